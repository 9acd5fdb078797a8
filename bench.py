"""Benchmark of the RadRHD_solver hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): one RHLLC hydro step (face fluxes + conservative update +
con2prim with the PhysPressureFix fallback, FP64) on the coupled-jet mesh:
cube [-1,1]^3 as 96^3 hexes x 6 Kuhn tets = 5,308,416 cells, 10,672,128 faces
(vertices jittered +-0.15h, seeded), ambient rho=1, p=1e-3, v=0, Gamma=4/3,
inflow nozzle r<0.1 at z=-1 (rho=0.01, W=7 along +z, p=1e-3), transmissive
walls, tau = 0.3 h_min / c.  Synthetic, seeded; no dataset exists for this.

value = cell-updates/s with the state resident in HBM (CUDA events on the
solver's stream, max over ranks); e2e = the same through the C ABI drop-in
rrhd_hydro_step_host with host (pinned) buffers: H2D of W,U + step + D2H of W,U
every step.  The state (2 x 425 MB) is larger than L2, so no flush is needed.

--impl reference: the reference's own CPU implementation of the same step
(rhllc::Hllc3dStab compiled from its sources with -Ofast -fopenmp, oracle/_ref)
on all host cores; rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s (RHLLC+con2prim); scatter cell-dir/s; chosen vs plain form"
UNIT = "cell-updates/s"
NHEX = 96
GAMMA = 4.0 / 3.0
CFL = 0.3
INFLOW = [0.01, 0.0, 0.0, float(np.sqrt(1.0 - 1.0 / 49.0)), 1e-3]
DATA = "synthetic (seeded Kuhn mesh, jet initial state)"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


JET_MESH = dict(lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, inflow_radius=0.1, inflow_code=-3)


def make_jet(n=None, seed=2024, independent=False):
    """The jet mesh and its ambient primitive state.  independent=True builds the
    mesh with the oracle's numpy generator (bit-identical to the library's, pinned
    by tests/test_oracle_kuhn.py), so that the CPU reference arm never loads the
    CUDA library."""
    n = n or NHEX
    if independent:
        from oracle import kuhn as K
        m = K.kuhn_box(n, n, n, seed=seed, **JET_MESH)
    else:
        from radrhd_solver_b200 import mesh as M
        m = M.kuhn_box(n, n, n, seed=seed, **JET_MESH)
    W = np.zeros((m.n_cells, 5))
    W[:, 0] = 1.0
    W[:, 4] = 1e-3
    return m, W


def bench_config(m, ws):
    """The workload description both arms print (identical keys and values)."""
    return {"workload": f"coupled-jet mesh {NHEX}^3x6 tets: RHLLC flux + update + con2prim step",
            "cells": m.n_cells, "faces": m.n_faces, "gamma": GAMMA, "tau": CFL * m.h_min,
            "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
            "l2": f"state 2 x {80 * m.n_cells / 1e6:.0f} MB, L2 126 MB: "
                  + ("larger than L2, no flush" if 80 * m.n_cells > 126e6 else "fits in L2 (a small case)")}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        rows = []
        for ln in (self.out or "").strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 8:
                rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, ws: int, device: str) -> float:
    """The slowest rank's value (job time = max over ranks); every rank takes the
    same collective step."""
    if ws <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, ws: int, steps: int, ms_max: float) -> float:
    """Whole-job units per second: every replica processes units_per_rank per step."""
    return ws * units_per_rank * steps / (ms_max / 1e3)


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_steps(m, W, U, steps, threads, bc_u):
    """Times `steps` reference hydro steps on the host; returns seconds per step and kind."""
    import oracle
    variant = REF_VARIANT
    if oracle.have_ref(variant):
        h = oracle.HydroRef(m, variant)
        h.set_bc(-3, 1, np.array(INFLOW), bc_u)
        h.set_state(W, U)
        tau = CFL * m.h_min
        h.step(tau, threads)  # first touch
        t0 = time.perf_counter()
        for _ in range(steps):
            h.step(tau, threads)
        dt = (time.perf_counter() - t0) / steps
        h.close()
        return dt, "reference"
    # the C restatement when the reference could not be built
    bc = {-3: (1, np.array(INFLOW), bc_u)}
    tau = CFL * m.h_min
    t0 = time.perf_counter()
    for _ in range(steps):
        U, W, _, _, _ = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA, bc=bc, nthreads=threads)
    return (time.perf_counter() - t0) / steps, "port"


REF_VARIANT = "hydro_ideal_4_3_fast"


def inflow_conservative():
    """Conservative inflow state (rhllc::GetConvValue, solvers/rhllc/src/rhllc_flux.cpp:7-16)
    for the CPU legs: the reference's own function where it was built, else the oracle's."""
    import oracle
    u = np.zeros(5)
    w = np.array(INFLOW)
    lib = oracle.ref(REF_VARIANT)
    if lib is not None:
        lib.ref_p2c_plain(w.ctypes.data, u.ctypes.data, 1)
        return u
    e = oracle.loader.OrcEos(1, GAMMA)
    oracle.port().orc_p2c_plain(ctypes.byref(e), w.ctypes.data, u.ctypes.data)
    return u


def run_reference(args):
    """The reference's CPU hydro step (rhllc::Hllc3dStab from its own sources) on the
    same mesh, state and time step as the GPU arm; this process never loads the CUDA
    library (mesh from the oracle's generator, states from the reference's prim->cons)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    m, W = make_jet(independent=True)
    W, U = _p2c_fast(W)
    threads = cpu_threads()
    bc_u = inflow_conservative()
    dt, kind = reference_steps(m, W, U, max(1, args.steps), threads, bc_u)
    v = m.n_cells / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": bench_config(m, args.gpus),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{args.steps} full steps of the {m.n_cells}-cell mesh"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _p2c_fast(W):
    """prim->cons (GetConvValueStab) of the uniform ambient state, computed once by
    the reference's own function where it was built (else the oracle's) and
    repeated over the mesh."""
    import oracle
    if oracle.have_ref(REF_VARIANT):
        Wu, Uu = oracle.ref_p2c(W[:1], REF_VARIANT)
    else:
        Wu, Uu = oracle.port_p2c(W[:1], 1, GAMMA)
    return np.repeat(Wu, len(W), 0), np.repeat(Uu, len(W), 0)


def profile_figure(name, key="traffic_bytes_per_launch"):
    """A figure recorded from an ncu capture in profiles/<name> as a line "key: value"."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for ln in open(p):
            if ln.strip().startswith(key + ":"):
                return float(ln.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


def _time(fn, reps, stream, warm=2):
    import torch
    for _ in range(warm):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def scatter_component(dev, nhex=48, M=256, groups=1, kind=0, sigma=0.5, reps=5, fp64=True):
    """Scattering integral + moments, plain FP64 and tensor-core forms.
    nhex=48, M=256, groups=1: 663,552 cells x 256 directions (lognormal(0,0.5) x
    exp(-|x|^2/0.2)); inputs 0.68 GB (FP32) / 1.36 GB (FP64) > L2, no flush."""
    import torch
    from radrhd_solver_b200 import _lib as L
    from radrhd_solver_b200 import illum
    from radrhd_solver_b200 import mesh as Mm
    m = Mm.kuhn_box(nhex, nhex, nhex, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, seed=7)
    rows = m.n_cells * groups
    d = Mm.fibonacci_directions(M)
    dg = illum.DirectionGrid(d, dev)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    centers = torch.tensor(m.cell_center, device=f"cuda:{dev}")
    out = {"workload": f"{m.n_cells} cells x {groups} groups x {M} directions", "rows": rows, "M": M}
    flop = 2.0 * rows * M * (M + 10)  # algorithmic: S plus the 10 moment columns
    cd = rows * M
    I32 = torch.empty(rows, M, dtype=torch.float32, device=f"cuda:{dev}")
    L.check(L.lib.rrhd_fill_intensity_f32(I32.data_ptr(), rows, M, groups, kind, sigma, centers.data_ptr(), 11, sp))
    if fp64:
        I64 = torch.empty(rows, M, dtype=torch.float64, device=f"cuda:{dev}")
        L.check(L.lib.rrhd_fill_intensity_f64(I64.data_ptr(), rows, M, groups, kind, sigma, centers.data_ptr(), 11, sp))
        S64 = torch.empty_like(I64)
        E = torch.empty(rows, dtype=torch.float64, device=I64.device)
        F = torch.empty(rows, 3, dtype=torch.float64, device=I64.device)
        T = torch.empty(rows, 3, 3, dtype=torch.float64, device=I64.device)
        for name, fn in (("fp64_exact", L.lib.rrhd_scatter_fp64), ("fp64_fma", L.lib.rrhd_scatter_fp64_fma)):
            def run(fn=fn):
                L.check(fn(dg.handle, I64.data_ptr(), S64.data_ptr(), rows, sp))
                L.check(L.lib.rrhd_moments_fp64(dg.handle, I64.data_ptr(), E.data_ptr(), F.data_ptr(), T.data_ptr(),
                                                rows, sp))
            ms = _time(run, reps, stream)
            out[name] = {"ms": ms, "cell_dir_per_s": cd / (ms / 1e3), "tflops": flop / (ms / 1e3) / 1e12}
        # the same S and moments through the rank-7 Thomson identity (O(M) per row)
        mom64 = torch.empty(rows, 16, dtype=torch.float64, device=I64.device)

        def run_lr64():
            L.check(L.lib.rrhd_scatter_lowrank(dg.handle, I64.data_ptr(), S64.data_ptr(), mom64.data_ptr(), rows, 1,
                                               L.RRHD_RAD_FP64, sp))
        ms = _time(run_lr64, reps, stream)
        out["fp64_lowrank"] = {"ms": ms, "cell_dir_per_s": cd / (ms / 1e3),
                               "gbs": (rows * M * 16 + rows * 128) / (ms / 1e3) / 1e9}
        del I64, S64, mom64
    S32 = torch.empty_like(I32)
    mom = torch.empty(rows, 16, dtype=torch.float32, device=I32.device)

    def run_lr32():
        L.check(L.lib.rrhd_scatter_lowrank(dg.handle, I32.data_ptr(), S32.data_ptr(), mom.data_ptr(), rows, 1,
                                           L.RRHD_RAD_FP32, sp))
    ms = _time(run_lr32, reps, stream)
    out["fp32_lowrank"] = {"ms": ms, "cell_dir_per_s": cd / (ms / 1e3),
                           "gbs": (rows * M * 8 + rows * 64) / (ms / 1e3) / 1e9}
    for form in ("f16x3", "bf16x3", "f16"):
        tc = illum.ScatterTC(dg, form)

        def run(tc=tc):
            L.check(L.lib.rrhd_scatter_tc_run(tc._h, I32.data_ptr(), S32.data_ptr(), mom.data_ptr(), rows, sp))
        ms = _time(run, reps, stream)
        tc.check()
        nbytes = rows * M * 8 + rows * 64
        out["tc_" + form] = {"ms": ms, "cell_dir_per_s": cd / (ms / 1e3), "tflops": flop / (ms / 1e3) / 1e12,
                             "gbs": nbytes / (ms / 1e3) / 1e9}
        tc.close()
    dg.close()
    return out


def scatter_scale_component(dev, cells=2_000_000, M=512, groups=16, reps=3, sample=65536):
    """Config 2: 2M cells x 512 Fibonacci directions x 16 frequency groups in one launch
    (rows = cell x group); I = 10^(-6 + 6g/15) lognormal(0, 1) (seeded), values over
    ~12 decades.  Tensor-core forms timed on all 32M rows (I and S 64 GB each, FP32);
    errors against the direct FP64 contraction on a seeded sample of rows and against
    the FP64 low-rank (rank-7 Thomson) values on every row."""
    import torch
    from radrhd_solver_b200 import _lib as L
    from radrhd_solver_b200 import illum
    from radrhd_solver_b200 import mesh as Mm
    torch.cuda.empty_cache()
    rows = cells * groups
    d = Mm.fibonacci_directions(M)
    dg = illum.DirectionGrid(d, dev)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    I32 = torch.empty(rows, M, dtype=torch.float32, device=f"cuda:{dev}")
    L.check(L.lib.rrhd_fill_intensity_f32(I32.data_ptr(), rows, M, groups, 1, 1.0, None, 23, sp))
    S32 = torch.empty_like(I32)
    gen = torch.Generator(device="cpu").manual_seed(5)
    idx = torch.randperm(rows, generator=gen)[:sample].sort().values.to(f"cuda:{dev}")
    I64 = I32[idx].double()
    S64 = torch.empty_like(I64)
    L.check(L.lib.rrhd_scatter_fp64(dg.handle, I64.data_ptr(), S64.data_ptr(), sample, sp))
    flop = 2.0 * rows * M * M
    out = {"workload": f"{cells} cells x {groups} groups x {M} directions, one launch", "rows": rows,
           "error_sample_rows": sample}
    for form in ("bf16x3", "f16x3", "f16"):
        tc = illum.ScatterTC(dg, form)

        def run(tc=tc):
            L.check(L.lib.rrhd_scatter_tc_run(tc._h, I32.data_ptr(), S32.data_ptr(), None, rows, sp))
        ms = _time(run, reps, stream, warm=1)
        tc.check()
        rel = ((S32[idx].double() - S64).abs() / S64.abs()).flatten()
        mx_all, rms_all = illum.LowRankError(dg, I32, S32, stream=sp)
        out["tc_" + form] = {"ms": ms, "row_dir_per_s": rows * M / (ms / 1e3), "tflops": flop / (ms / 1e3) / 1e12,
                             "max_rel_err": float(rel.max()), "rms_rel_err": float(rel.pow(2).mean().sqrt()),
                             "all_rows_lowrank": {"max_rel_err": mx_all, "rms_rel_err": rms_all}}
        tc.close()
    def run_lr():
        L.check(L.lib.rrhd_scatter_lowrank(dg.handle, I32.data_ptr(), S32.data_ptr(), None, rows, 1,
                                           L.RRHD_RAD_FP32, sp))
    ms = _time(run_lr, reps, stream, warm=1)
    rel = ((S32[idx].double() - S64).abs() / S64.abs()).flatten()
    out["fp32_lowrank"] = {"ms": ms, "row_dir_per_s": rows * M / (ms / 1e3),
                           "max_rel_err": float(rel.max()), "rms_rel_err": float(rel.pow(2).mean().sqrt())}
    del I32, S32, I64, S64
    dg.close()
    torch.cuda.empty_cache()
    return out


def c2p_component(dev, n=8_000_000, epochs=8, reps=5):
    """Config 3: 8M states (rho, p/rho, W log-uniform; isotropic v; Gamma 4/3),
    network trained on the first 4M, plain vs learned-guess con2prim timed on the
    other 4M (inputs 160 MB U + 160 MB W > L2)."""
    import torch
    from radrhd_solver_b200 import _lib as L
    from radrhd_solver_b200 import rhllc
    from radrhd_solver_b200.c2p_mlp import LearnedGuess
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    W = torch.empty(n, 5, dtype=torch.float64, device=f"cuda:{dev}")
    L.check(L.lib.rrhd_fill_c2p_states(W.data_ptr(), n, 2024, sp))
    U = torch.empty_like(W)
    rhllc.GetConvValueStab(W, U, eos=1, gamma=GAMMA, stream=sp)
    h = n // 2
    Utr, ptr_ = U[:h].contiguous(), W[:h, 4].contiguous()
    Ute = U[h:].contiguous()
    net = LearnedGuess(device=dev, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = net.train(Utr, ptr_, epochs=epochs, batch=4096, lr=2e-3, seed=3, stream=sp)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    out = {"workload": f"{n} states (train {h}, test {n - h})", "train_s": t_train,
           "train_loss_first_last": [float(hist[0]), float(hist[-1])]}

    def both_forms(Ut):
        """plain and learned-guess con2prim of the states Ut (each timed call restores U)."""
        k = Ut.shape[0]
        Wo, Uw = torch.empty_like(Ut), torch.empty_like(Ut)
        st_box, res = {}, {}

        def plain():
            Uw.copy_(Ut)
            st_box["p"] = L.C2pStats()
            L.check(L.lib.rrhd_con2prim_batch_stats(1, GAMMA, Uw.data_ptr(), Wo.data_ptr(), None, k, 1,
                                                    ctypes.byref(st_box["p"]), sp))

        def learned():
            Uw.copy_(Ut)
            st_box["l"] = L.C2pStats()
            st_box["nb"] = ctypes.c_int64()
            L.check(L.lib.rrhd_con2prim_batch_mlp(net.handle, 1, GAMMA, Uw.data_ptr(), Wo.data_ptr(), None, k, 1, 8,
                                                  ctypes.byref(st_box["l"]), ctypes.byref(st_box["nb"]), None, sp))

        def copy_only():
            Uw.copy_(Ut)
        t_copy = _time(copy_only, reps, stream)
        for name, fn in (("plain_guess", plain), ("learned_guess", learned)):
            ms = _time(fn, reps, stream) - t_copy
            key = "p" if name == "plain_guess" else "l"
            st = st_box[key]
            res[name] = {"ms": ms, "states_per_s": k / (ms / 1e3), "newton_iters_per_state": st.newton_iters / k,
                         "max_iters": st.max_iters, "pressure_fix_fallbacks": st.n_fallback, "failed": st.n_failed}
            if key == "l":
                res[name]["guess_fallbacks"] = st_box["nb"].value
        return res

    out.update(both_forms(Ute))
    # the fast-flow part of the same held-out states, where the reference guess is poorest
    v2 = (W[h:, 1:4] ** 2).sum(1)
    hi = (1.0 / torch.sqrt(1.0 - v2)) >= 10.0
    sub = both_forms(Ute[hi].contiguous())
    out["lorentz_ge_10"] = {"states": int(hi.sum().item()), **sub}
    net.close()
    return out


EM_JET = (1.0, 10.0, float(np.pi), 1.0)  # temp_coef, a_R, pi, kRadiation in code units: T = p / rho, B = a_R T^4 / pi


def coupled_component(dev, m, W, steps=100, warm=1, M=256, G=4, train_epochs=2, forms=("plain", "chosen"),
                      batch=(128, 256), item_geometry=True):
    """Config-4 coupled radiation-hydro jet step (radRHD_main.cpp:96-139) on the
    benchmark mesh: hydro step, opacities alpha = rho, betta = 0.5 rho, emission
    Q = a_R T^4 / pi / G per grey group, sweep of M directions x G groups,
    4-force + source con2prim, scattering integral + moments.  Plain form: FP64
    sweep, FP64 scattering (one FMA per term), reference con2prim guess.  Chosen
    form: mixed-precision sweep (FP64 arithmetic and face values, FP32 intensity
    and scattering integral; with item_geometry, each (cell, direction) item's
    geometry precomputed at setup and streamed), tensor-core F16X3 scattering,
    learned con2prim guess trained on the plain run's own states.  "plain_lowrank" / "chosen_lowrank": the
    same with the scattering through the rank-7 Thomson identity (FP64 arithmetic).
    All forms start from the same state; the intensity arrays (N*G*M = 5.4e9
    values) are far larger than L2."""
    import torch
    from radrhd_solver_b200 import illum, rad_rhd, rhllc
    from radrhd_solver_b200 import mesh as Mm
    from radrhd_solver_b200.c2p_mlp import LearnedGuess
    d = Mm.fibonacci_directions(M)
    tau = CFL * m.h_min
    out = {"workload": f"coupled jet {m.n_cells} cells x {M} directions x {G} groups", "cells": m.n_cells,
           "directions": M, "groups": G, "emission": {"temp_coef": EM_JET[0], "a_R": EM_JET[1], "rad_unit": EM_JET[3]},
           "tau": tau, "steps": steps}
    states = {}
    net = None
    for form in forms:
        fp64 = form.startswith("plain")
        torch.cuda.empty_cache()
        g = rhllc.Grid(m, eos=rhllc.EOS_IDEAL, gamma=GAMMA, device=dev)
        g.set_boundary(-3, rhllc.BC_FIXED, INFLOW)
        g.set_state_prim(W)
        dg = illum.DirectionGrid(d, dev)
        t0 = time.perf_counter()
        geo = item_geometry and not fp64
        sw = illum.TransportSweep(g, dg, groups=G, precision="fp64" if fp64 else "mixed",
                                  dirs_per_batch=batch[0] if fp64 else batch[1], item_geometry=geo)
        t_plan = time.perf_counter() - t0
        if not fp64 and net is None and "plain_dump" in states:
            Wp, Up = states["plain_dump"]
            net = LearnedGuess(device=dev, seed=1)
            Ut = torch.tensor(Up, device=f"cuda:{dev}")
            pt = torch.tensor(Wp[:, 4], device=f"cuda:{dev}")
            net.train(Ut, pt, epochs=train_epochs, batch=4096, lr=2e-3, seed=3)
            del Ut, pt
        step = rad_rhd.RadRHDStep(sw, absorption=1.0, scattering=0.5, em=rad_rhd.emission(*EM_JET),
                                  scatter="lowrank" if form.endswith("_lowrank") else ("fp64" if fp64 else "f16x3"),
                                  guess=None if fp64 else net)
        stream = torch.cuda.ExternalStream(g.stream)
        warm_stats = [step(tau, stats=True) for _ in range(warm)]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fails = [0, 0, 0]  # hydro cells failed after the fallback, hydro fallbacks, source con2prim failures
        for _ in range(steps):
            hs, ss = step(tau, stats=True)  # reads the step's counters back (one sync per step)
            fails[0] += hs.n_failed
            fails[1] += hs.n_fallback
            fails[2] += ss.n_failed
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        ph = step.phase_ms()
        levels, biggest = sw.plan_info()
        # the reduced-precision scattering of the last step against FP64 from the same intensity
        scat_err = None
        if not fp64:
            emax, erms, emom = step.scatter_error(65536)
            scat_err = {"sample_cells": 65536, "max_rel": emax, "rms_rel": erms, "moments_max": emom}
        Wg, Ug = g.get_state()
        states[form] = Ug
        if form == "plain":
            states["plain_dump"] = (Wg, Ug)
        bio = 8 if fp64 else 4  # bytes per intensity / scattering value; face values are double
        sweep_alg = (2.0 * m.n_cells * bio + 2.0 * m.n_faces * 8) * M * G + m.n_cells * (20 * 8 + 32.0)
        if geo:
            sweep_alg += 16.0 * m.n_cells * M  # the item-geometry stream
        out[form] = {"dirs_per_batch": batch[0] if fp64 else batch[1], "item_geometry": geo, "ms_per_step": ms, "steps_per_s": 1e3 / ms, "cell_updates_per_s": m.n_cells / (ms / 1e3),
                     "cell_dir_group_per_s": m.n_cells * M * G / (ms / 1e3), "phase_ms_last_step": ph,
                     "sweep_levels": levels, "largest_level": biggest, "plan_build_s": t_plan,
                     "scatter_op_error": scat_err,
                     "sweep_alg_gbs": sweep_alg / (ph["sweep"] / 1e3) / 1e9,
                     "source_c2p": {"newton_iters_per_state_last_step": ss.newton_iters / m.n_cells,
                                    "failed_all_steps": fails[2]},
                     "hydro": {"n_fallback_all_steps": fails[1], "n_failed_all_steps": fails[0]},
                     "warmup_failures": [[h.n_failed, s_.n_failed] for h, s_ in warm_stats]}
        g.close()
        dg.close()
        del step, sw
    if net is not None:
        net.close()
    if "plain" in states and "chosen" in states:
        up, uc = states["plain"], states["chosen"]
        # per cell: D and E relative to themselves, the momentum relative to the cell's E
        E = np.abs(up[:, 4])
        du = max(float(np.max(np.abs(uc[:, [0, 4]] - up[:, [0, 4]]) / np.abs(up[:, [0, 4]]))),
                 float(np.max(np.abs(uc[:, 1:4] - up[:, 1:4]) / E[:, None])))
        out["state_max_rel_diff_per_cell"] = du
        out["chosen_vs_plain"] = out["plain"]["ms_per_step"] / out["chosen"]["ms_per_step"]
    return out


def sweep_component(dev, nhex=32, M=256, G=4, reps=3, precisions=("fp64", "fp32")):
    """Standalone transport sweep (rrhd_sweep) on the jet mesh with seeded
    opacities and sources: alpha log-uniform [0.1, 30], betta = alpha / 2, Q and S
    log-uniform; the unit is one (cell, direction) pair with all G groups."""
    import torch
    from radrhd_solver_b200 import illum, rhllc
    from radrhd_solver_b200 import mesh as Mm
    m, _ = make_jet(nhex)
    d = Mm.fibonacci_directions(M)
    out = {"workload": f"sweep {m.n_cells} cells x {M} directions x {G} groups", "cells": m.n_cells, "faces": m.n_faces}
    for prec in precisions:
        torch.cuda.empty_cache()
        g = rhllc.Grid(m, eos=rhllc.EOS_IDEAL, gamma=GAMMA, device=dev)
        dg = illum.DirectionGrid(d, dev)
        t0 = time.perf_counter()
        sw = illum.TransportSweep(g, dg, groups=G, precision=prec)
        t_plan = time.perf_counter() - t0
        dt = torch.float64 if prec == "fp64" else torch.float32
        gen = torch.Generator(device=f"cuda:{dev}").manual_seed(5)
        rnd = lambda *shape, lo, hi: (10 ** (lo + (hi - lo) * torch.rand(*shape, generator=gen, device=f"cuda:{dev}",
                                                                        dtype=torch.float64))).to(dt)
        alpha = rnd(m.n_cells, lo=-1, hi=1.5)
        betta = (0.5 * alpha).contiguous()
        Q = rnd(m.n_cells, G, lo=-2, hi=0)
        S = rnd(m.n_cells * G, M, lo=-3, hi=-1)
        I = torch.empty_like(S)
        torch.cuda.synchronize()
        stream = torch.cuda.ExternalStream(g.stream)
        ms = _time(lambda: illum.CalculateIllum(sw, alpha, betta, Q, S, I), reps, stream, warm=1)
        levels, biggest = sw.plan_info()
        bpv = 8 if prec == "fp64" else 4
        alg = (2.0 * m.n_cells + 2.0 * m.n_faces) * M * G * bpv + m.n_cells * (20 * bpv + 32.0)
        out[prec] = {"ms": ms, "cell_dir_per_s": m.n_cells * M / (ms / 1e3), "levels": levels,
                     "largest_level": biggest, "plan_build_s": t_plan, "alg_gbs": alg / (ms / 1e3) / 1e9}
        del alpha, betta, Q, S, I
        g.close()
        dg.close()
    return out


def compton_component(dev, cells=1184, M=256, reps=3, cpu_cells=8):
    """Frequency-coupled Compton scattering over the 100-bin spectrum
    (rrhd_compton_full_spectrum) on seeded intensities [cells][M][100] (lognormal
    times a smooth spectral shape) and velocities cycling through 0, 1e-6, 1e-5,
    0.3, 0.9 and 0.99 c.  The unit is one term (cell, output direction, frequency,
    incoming direction): cells x M x 100 x M per call.  The first cpu_cells cells
    also run through the reference's own kernel source compiled for the host
    (oracle/_ref, all host threads; the oracle port where that is absent), which
    gives the CPU rate and the parity of the timed result on those cells."""
    import torch
    from radrhd_solver_b200 import illum
    from radrhd_solver_b200 import mesh as Mm
    d = Mm.fibonacci_directions(M)
    dg = illum.DirectionGrid(d, dev)
    gen = torch.Generator(device=f"cuda:{dev}").manual_seed(31)
    f = torch.arange(100, device=f"cuda:{dev}", dtype=torch.float64)
    shape = torch.exp(-((f - 60.0) / 25.0) ** 2) + 0.05
    I = torch.exp(0.5 * torch.randn(cells, M, 100, generator=gen, device=f"cuda:{dev}", dtype=torch.float64)) * shape
    u = torch.randn(cells, 3, generator=gen, device=f"cuda:{dev}", dtype=torch.float64)
    speeds = torch.tensor([0.0, 1e-6, 1e-5, 0.3, 0.9, 0.99], device=f"cuda:{dev}", dtype=torch.float64)
    vel = u / u.norm(dim=1, keepdim=True) * speeds[torch.arange(cells, device=f"cuda:{dev}") % 6][:, None]
    S = torch.empty(cells, M, 100, dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    ms = _time(lambda: illum.FullSpectrumScattering(dg, I, vel, S=S), reps, stream, warm=1)
    terms = float(cells) * M * 100 * M
    out = {"workload": f"full-spectrum Compton scattering {cells} cells x {M} directions x 100 bins",
           "ms": ms, "terms_per_s": terms / (ms / 1e3), "unit": "terms/s",
           "l2": f"I {I.numel() * 8 / 1e6:.0f} MB > L2; the kernel is FP64-bound, not memory-bound"}
    # single frequency (rrhd_compton_spectrum): the same intensities as 100 x cells rows at one frequency
    I1 = I.permute(0, 2, 1).reshape(cells * 100, M).contiguous()
    v1 = vel.repeat_interleave(100, dim=0).contiguous()
    S1 = torch.empty_like(I1)
    ms1 = _time(lambda: illum.SpectrumScattering(dg, I1, v1, 4.2e20, S=S1), reps, stream, warm=1)
    out["single_frequency"] = {"workload": f"{cells * 100} cells x {M} directions at 4.2e20 Hz", "ms": ms1,
                               "terms_per_s": float(cells) * 100 * M * M / (ms1 / 1e3)}
    del I1, v1, S1
    import oracle
    threads = cpu_threads()
    Ih, vh, Sh = I[:cpu_cells].cpu().numpy(), vel[:cpu_cells].cpu().numpy(), S[:cpu_cells].cpu().numpy()
    t0 = time.perf_counter()
    So = oracle.ref_compton(Ih, vh, d.dirs, d.areas, d.full_area, nthreads=threads)
    kind = "reference"
    if So is None:
        So = oracle.port_compton(Ih, vh, d.dirs, d.areas, d.full_area, nthreads=threads)
        kind = "port"
    dt = time.perf_counter() - t0
    nz = So != 0
    out["max_rel_err_vs_cpu"] = float(np.max(np.abs(Sh[nz] - So[nz]) / np.abs(So[nz])))
    out["cpu_baseline"] = {"value": cpu_cells * M * 100.0 * M / dt, "unit": "terms/s", "cores": threads,
                           "kind": kind, "sample": f"{cpu_cells} cells of the same workload"}
    out["vs_cpu"] = out["terms_per_s"] / out["cpu_baseline"]["value"]
    dg.close()
    return out


def ray_component(dev, n_box=48, n_sphere=64, frame=11, reps=3, cpu_rays=1500):
    """Image-plane ray tracing (rrhd_ray_trace): one frame of 600 x 300 rays against the
    triangulated boundary of a box around the scene plus a sphere around the accretor
    (tests/cases.py ray_surface); the unit is one ray resolved against the whole surface
    (pairs_per_s: the same as ray-triangle pairs of the reference's brute-force loop).  The
    reference's own kernel sources compiled for the host time a sample of the rays."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cases import ray_surface
    from radrhd_solver_b200 import ray_tracing as RT
    ids, abc = ray_surface(n_box, n_sphere)
    rt = RT.RayTracer(RT.face_cells(ids, abc), dev)
    rays_h = RT.MakeRays(frame)
    rays = torch.tensor(rays_h, device=f"cuda:{dev}")
    codes = torch.empty(len(rays_h), dtype=torch.int32, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    out = {"workload": f"ray tracing {len(rays_h)} rays x {len(ids)} triangles", "unit": "rays/s"}
    pairs = float(len(rays_h)) * len(ids)
    for mode, name in ((RT.SURFACE, "surface"), (RT.ROCHE, "roche"), (RT.INNER, "inner")):
        ms = _time(lambda: rt.trace(rays, mode, codes), reps, stream, warm=1)
        out[name] = {"ms": ms, "rays_per_s": len(rays_h) / (ms / 1e3), "pairs_per_s": pairs / (ms / 1e3)}
    import oracle
    sample = rays_h[:: len(rays_h) // cpu_rays][:cpu_rays]
    t0 = time.perf_counter()
    got = oracle.ref_ray(RT.SURFACE, sample, ids, abc, nthreads=cpu_threads())
    kind = "reference"
    if got is None:
        got = oracle.port_ray_trace(RT.SURFACE, sample, ids, abc, nthreads=cpu_threads())
        kind = "port"
    dt = time.perf_counter() - t0
    gpu = rt.trace(rays, RT.SURFACE, codes).cpu().numpy()[:: len(rays_h) // cpu_rays][:cpu_rays]
    out["codes_equal_to_cpu"] = bool(np.array_equal(gpu, got))
    out["cpu_baseline"] = {"value": len(sample) / dt, "unit": "rays/s", "cores": cpu_threads(),
                           "kind": kind, "sample": f"{len(sample)} rays of the frame, surface mode"}
    out["vs_cpu"] = out["surface"]["rays_per_s"] / out["cpu_baseline"]["value"]
    rt.close()
    return out


def run_ours(args):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local
    torch.cuda.set_device(dev)
    from radrhd_solver_b200 import _lib as L
    from radrhd_solver_b200 import rhllc

    m, W = make_jet()
    g = rhllc.Grid(m, eos=rhllc.EOS_IDEAL, gamma=GAMMA, device=dev, cells_per_block=args.cpb)
    layout = g.layout_info()
    g.set_boundary(-3, rhllc.BC_FIXED, INFLOW)
    g.set_state_prim(W)
    tau = CFL * m.h_min
    stream = torch.cuda.ExternalStream(g.stream)
    for _ in range(args.warmup):
        L.check(L.lib.rrhd_hydro_step(g.handle, tau, None))
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # device-resident timing
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with Clocks(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            L.check(L.lib.rrhd_hydro_step(g.handle, tau, None))
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    st = L.StepStats()
    L.check(L.lib.rrhd_hydro_step(g.handle, tau, ctypes.byref(st)))
    ms = max_over_ranks(ms, ws, f"cuda:{dev}")
    per_step = ms / args.steps
    value = job_throughput(m.n_cells, ws, args.steps, ms)

    # e2e through the host-buffer drop-in
    Wh = torch.empty((m.n_cells, 5), dtype=torch.float64).pin_memory()
    Uh = torch.empty((m.n_cells, 5), dtype=torch.float64).pin_memory()
    L.check(L.lib.rrhd_get_state(g.handle, Wh.data_ptr(), Uh.data_ptr(), 5, L.RRHD_HOST))
    e2e_steps = max(3, args.steps // 2)
    L.check(L.lib.rrhd_hydro_step_host(g.handle, tau, Wh.data_ptr(), Uh.data_ptr(), 5, None))
    barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        L.check(L.lib.rrhd_hydro_step_host(g.handle, tau, Wh.data_ptr(), Uh.data_ptr(), 5, None))
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e = max_over_ranks(e0.elapsed_time(e1), ws, f"cuda:{dev}")
    e2e_value = job_throughput(m.n_cells, ws, e2e_steps, ms_e)
    io_bytes = 80 * m.n_cells

    # e2e in the drop-in's resident mode: the host state uploaded once, every step reading
    # back its step scalars (max signal speed) as rhllc::Hllc3dStab must, the state written
    # back to the host buffers every SAVE steps (the save cadence of WriteSolution)
    SAVE = 10
    res_steps = max(SAVE, (args.steps // SAVE) * SAVE)
    stt = L.StepStats()
    barrier()
    e0.record(stream)
    L.check(L.lib.rrhd_set_state(g.handle, Wh.data_ptr(), Uh.data_ptr(), 5, L.RRHD_HOST))
    for k in range(res_steps):
        L.check(L.lib.rrhd_hydro_step(g.handle, tau, ctypes.byref(stt)))
        if (k + 1) % SAVE == 0:
            L.check(L.lib.rrhd_get_state(g.handle, Wh.data_ptr(), Uh.data_ptr(), 5, L.RRHD_HOST))
    e1.record(stream)
    torch.cuda.synchronize()
    ms_r = max_over_ranks(e0.elapsed_time(e1), ws, f"cuda:{dev}")
    e2e_res = {"value": job_throughput(m.n_cells, ws, res_steps, ms_r), "unit": UNIT,
               "h2d_bytes_per_step": io_bytes / res_steps, "d2h_bytes_per_step": io_bytes / SAVE + 32,
               "save_every_steps": SAVE, "steps": res_steps}

    # roofline of the fused step kernel (the only kernel in the step)
    alg_bytes = 185.0 * m.n_cells + 40.0 * m.n_faces
    achieved = alg_bytes / (per_step / 1e3) / 1e9
    pk = peaks()
    peak = pk["hbm_gbs"] if pk else 6650.0
    traffic = profile_figure("hydro_step_jet96.md") if NHEX == 96 else None
    fp64_pipe = profile_figure("hydro_step_jet96.md", "fp64_pipe_active_pct")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": bench_config(m, ws),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "measured" if pk else "fallback",
                         "algorithmic_bytes_per_cell_update": alg_bytes / m.n_cells,
                         # the bound that binds: FP64 dependency chains (ncu, 64^3 capture of the same kernel)
                         "fp64_pipe_active_pct": fp64_pipe,
                         # faces between two CTA blocks are fluxed by both (lists padded to even lengths)
                         "face_flux_evaluations_per_face": layout["face_entries"] / layout["faces"],
                         "cells_per_block": layout["cells_per_block"]},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
            "e2e_resident": e2e_res,
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "step_stats": {"max_speed": st.max_speed, "n_fallback": st.n_fallback, "n_failed": st.n_failed}}
    g.close()
    if rank == 0 and not args.no_coupled:
        line["coupled"] = coupled_component(dev, m, W, steps=args.coupled_steps,
                                            batch=tuple(int(x) for x in args.coupled_batch.split(",")),
                                            item_geometry=bool(args.coupled_item_geometry))
    if rank == 0 and not args.no_cpu:
        import oracle
        threads = cpu_threads()
        Wg = W.copy()
        Wg, Ug = _p2c_fast(Wg)
        dt, kind = reference_steps(m, Wg, Ug, args.cpu_steps, threads, inflow_conservative())
        line["cpu_baseline"] = {"value": m.n_cells / dt, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"{args.cpu_steps} full steps of the {m.n_cells}-cell mesh"}
    if rank == 0 and not args.no_c2p:
        line["c2p"] = c2p_component(dev)
    if rank == 0 and not args.no_scatter:
        line["scatter"] = scatter_component(dev)
        sc = line["scatter"]
        if "fp64_fma" in sc:
            line.setdefault("chosen_vs_plain", {})["scatter_moments"] = sc["fp64_fma"]["ms"] / sc["tc_f16x3"]["ms"]
    if rank == 0 and not args.no_scatter:
        line["scatter_scale"] = scatter_scale_component(dev)
    if rank == 0 and not args.no_compton:
        line["compton"] = compton_component(dev)
    if rank == 0 and not args.no_ray:
        line["ray_tracing"] = ray_component(dev)
    if rank == 0 and "coupled" in line:
        line.setdefault("chosen_vs_plain", {})["coupled_step"] = line["coupled"]["chosen_vs_plain"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--nhex", type=int, default=96, help="hexes per axis (96 = the benchmark mesh)")
    ap.add_argument("--cpb", type=int, default=0, help="cells per CTA of the step kernel (0 = library default)")
    ap.add_argument("--no-scatter", action="store_true", help="skip the scattering component")
    ap.add_argument("--no-c2p", action="store_true", help="skip the con2prim (learned guess) component")
    ap.add_argument("--no-coupled", action="store_true", help="skip the coupled radiation-hydro step component")
    ap.add_argument("--coupled-steps", type=int, default=100, help="timed coupled steps per form")
    ap.add_argument("--scatter-only", type=int, default=0, metavar="NHEX",
                    help="only time the scattering component on an NHEX^3 x 6 mesh (profiling runs)")
    ap.add_argument("--sweep-only", type=int, default=0, metavar="NHEX",
                    help="only time the standalone sweep on an NHEX^3 x 6 jet mesh (profiling runs)")
    ap.add_argument("--sweep-prec", default="fp64,fp32", help="precisions of --sweep-only")
    ap.add_argument("--coupled-only", type=int, default=0, metavar="NHEX",
                    help="only time the coupled step on an NHEX^3 x 6 jet mesh (profiling runs)")
    ap.add_argument("--coupled-forms", default="plain,chosen", help="forms of --coupled-only")
    ap.add_argument("--coupled-batch", default="128,256", help="directions per sweep batch (plain,chosen)")
    ap.add_argument("--coupled-item-geometry", type=int, default=1,
                    help="chosen forms: stream the precomputed per-item sweep geometry (1) or not (0)")
    ap.add_argument("--c2p-only", type=int, default=0, metavar="STATES",
                    help="only time the con2prim component on STATES states (profiling runs)")
    ap.add_argument("--no-compton", action="store_true", help="skip the full-spectrum Compton component")
    ap.add_argument("--no-ray", action="store_true", help="skip the image-plane ray-tracing component")
    ap.add_argument("--ray-only", action="store_true", help="only time the image-plane ray tracing")
    ap.add_argument("--compton-only", type=int, default=0, metavar="CELLS",
                    help="only time the full-spectrum Compton scattering on CELLS cells")
    ap.add_argument("--compton-m", type=int, default=256, help="directions of --compton-only")
    ap.add_argument("--scale-only", type=int, default=0, metavar="CELLS",
                    help="only time the scattering-at-scale component on CELLS cells (profiling runs)")
    args = ap.parse_args()
    global NHEX
    NHEX = args.nhex
    if args.scatter_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(scatter_component(0, nhex=args.scatter_only, reps=args.steps)), flush=True)
        return
    if args.ray_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(ray_component(0, reps=args.steps)), flush=True)
        return
    if args.compton_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(compton_component(0, cells=args.compton_only, M=args.compton_m, reps=args.steps,
                                           cpu_cells=2)), flush=True)
        return
    if args.c2p_only or args.scale_only:
        import torch
        torch.cuda.set_device(0)
        if args.c2p_only:
            print(json.dumps(c2p_component(0, n=args.c2p_only, reps=args.steps)), flush=True)
        else:
            print(json.dumps(scatter_scale_component(0, cells=args.scale_only, reps=args.steps,
                                                     sample=min(65536, args.scale_only))), flush=True)
        return
    if args.coupled_only:
        import torch
        torch.cuda.set_device(0)
        m, W = make_jet(args.coupled_only)
        print(json.dumps(coupled_component(0, m, W, steps=args.coupled_steps,
                                           forms=tuple(args.coupled_forms.split(",")),
                                           batch=tuple(int(x) for x in args.coupled_batch.split(",")),
                                           item_geometry=bool(args.coupled_item_geometry))), flush=True)
        return
    if args.sweep_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(sweep_component(0, nhex=args.sweep_only, reps=args.steps,
                                         precisions=tuple(args.sweep_prec.split(",")))), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
