"""Test infrastructure: the oracle (the checker, never the product).

`port`  : oracle/_build/librrhd_oracle.so, the plain-C restatement (rrhd_oracle.c).
`ref(v)`: oracle/_ref/librrhd_ref_<v>.so, the reference compiled from its own
          sources by oracle/Makefile (present only where the reference source
          tree was available when it was built).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from .loader import (HydroRef, build_port, have_ref, port, port_c2p, port_flux, port_hydro_step,  # noqa: F401
                     port_moments, port_p2c, port_pressure_fix, port_rad_source, port_scatter, ref,
                     ref_c2p, ref_flux, ref_moments, ref_p2c, ref_pressure_fix, ref_rad_source, ref_scatter,
                     ref_variant_for, port_get_illum, port_get_rhs, port_recalc_illum, port_sweep, ref_get_illum,
                     ref_get_rhs, ref_recalc_illum, ref_rad_constants, sweep_neighbours, port_compton,
                     port_compton_frq, port_compton_frq_idx, ref_compton, N_FRQ,
                     port_compton_spectrum, ref_compton_spectrum, port_ray_trace, port_ray_make_rays,
                     ref_ray, ref_ray_make_rays, RAY_PIXELS)
from . import loader  # noqa: F401
