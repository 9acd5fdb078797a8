"""GPU pieces of the coupled step over ranks (rad_rhd_mpi.GpuParts: rrhd_rad_opacities, the
sweep of a rank's directions, the FP64 scattering integral and moments of its rows,
rrhd_rad_source_rows, rrhd_rad_source_con2prim), run by RadRHDStepMPI on a one-rank NCCL
group in a child process.  Bar: three steps equal the oracle's single-process composition of
the same steps within 1e-12 per cell (the hydro state) and the single-GPU plain coupled step
(rrhd_coupled_step) within 1e-12.  The split over two and three ranks is covered on CPU by
test_coupled_split_gloo.py (the same host logic, the oracle computing the pieces)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


def _one_rank():
    import torch
    import torch.distributed as dist
    sys.path[:0] = [ROOT, HERE]
    import test_coupled_split_gloo as T
    from radrhd_solver_b200 import illum, rad_rhd, rad_rhd_mpi, rhllc, rhllc_mpi
    from cases import JET_INFLOW
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:" + os.environ["SPLIT_PORT"], rank=0,
                            world_size=1)
    try:
        oracle, gamma, m, W0, U0, bc, d, tau = T._setup()
        em = rad_rhd.emission(*T.EM)

        def grid():
            g = rhllc.Grid(m, gamma=gamma)
            g.set_boundary(-3, rhllc.BC_FIXED, JET_INFLOW)
            g.set_state(W0, U0)
            return g

        g = grid()
        rhllc_mpi.InitMpiConfig(g)
        step = rad_rhd_mpi.RadRHDStepMPI(rad_rhd_mpi.GpuParts(g, d, T.G, T.A, T.B, em, gamma=gamma))
        for _ in range(T.STEPS):
            st = step(tau)
            assert st.n_failed == 0
        W, U = g.get_state()
        # the single-GPU plain coupled step
        g1 = grid()
        dg = illum.DirectionGrid(d)
        sw = illum.TransportSweep(g1, dg, groups=T.G, precision="fp64")
        one = rad_rhd.RadRHDStep(sw, absorption=T.A, scattering=T.B, em=em, scatter="fp64")
        for _ in range(T.STEPS):
            one(tau)
        W1, U1 = g1.get_state()
        Uo, Wo = T._composition(oracle, gamma, m, W0, U0, bc, d, tau)

        def err(Ua, Ub):  # per cell: D, E relative to themselves, S relative to E
            E = np.abs(Ub[:, 4])[:, None]
            return max(np.max(np.abs(Ua[:, [0, 4]] - Ub[:, [0, 4]]) / np.abs(Ub[:, [0, 4]])),
                       np.max(np.abs(Ua[:, 1:4] - Ub[:, 1:4]) / E))
        e_o, e_1 = err(U, Uo), err(U, U1)
        print(f"coupled-split one rank: vs oracle composition {e_o:.2e}, vs rrhd_coupled_step {e_1:.2e}")
        assert e_o <= 1e-12 and e_1 <= 1e-12
        assert np.max(np.abs(W[:, 1:4] - Wo[:, 1:4])) <= 1e-12
    finally:
        dist.destroy_process_group()
    print("coupled-split-ok")


def test_coupled_step_split_one_rank_nccl():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    env = dict(os.environ, SPLIT_PORT=str(port), NCCL_NVLS_ENABLE="0")
    code = ("import sys; sys.path[:0] = [%r, %r]; import test_gpu_coupled_split as t; t._one_rank()"
            % (ROOT, HERE))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    print(r.stdout[-1500:])
    assert r.returncode == 0 and "coupled-split-ok" in r.stdout, r.stdout[-2000:] + r.stderr[-3000:]
