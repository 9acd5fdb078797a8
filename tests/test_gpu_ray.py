"""Image-plane ray tracing on the GPU (rrhd_ray_trace, rrhd_ray_image) against the oracle's
restatement of the reference kernels and the golden fixture made by the reference's own
sources.  Bar: every intersection code identical (the distances are formed in the
reference's operation order without contraction, so the nearest-hit choice is the same),
on image planes (one direction: the binned path) and on rays of many directions (every
triangle tested).
The image is checked value for value and the light curve within 1e-13 relative (its sum
runs in another order than the reference's sequential loop)."""
import os

import numpy as np
import pytest
import torch

import oracle
from cases import ray_surface
from radrhd_solver_b200 import ray_tracing as RT

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("mode", [RT.SURFACE, RT.ROCHE, RT.INNER, RT.GRID])
def test_trace_full_frame_matches_oracle(mode):
    ids, abc = ray_surface(12, 16)
    rays = RT.MakeRays(11)
    want = oracle.port_ray_trace(mode, rays, ids, abc, nthreads=os.cpu_count() or 1)
    rt = RT.RayTracer(RT.face_cells(ids, abc))
    got = rt.trace(torch.tensor(rays, device="cuda")).cpu().numpy() if mode == RT.SURFACE else \
        rt.trace(torch.tensor(rays, device="cuda"), mode).cpu().numpy()
    codes, counts = np.unique(want, return_counts=True)
    print(f"\nmode {mode}: {len(codes)} distinct codes, misses {counts[codes == -1].sum() if -1 in codes else 0}")
    assert np.array_equal(got, want)
    rt.close()


def test_trace_rays_of_many_directions_match_oracle():
    """Rays that do not share one direction take the every-triangle path."""
    ids, abc = ray_surface(6, 8)
    rng = np.random.default_rng(12)
    o = rng.uniform([-0.2, -0.6, -0.5], [2.0, 0.6, 0.5], (20000, 3))
    target = rng.uniform([0.5, -0.3, -0.2], [1.3, 0.3, 0.2], (20000, 3))
    rays = np.concatenate([o, target - o], axis=1)
    rt = RT.RayTracer(RT.face_cells(ids, abc))
    for mode in (RT.SURFACE, RT.INNER):
        want = oracle.port_ray_trace(mode, rays, ids, abc, nthreads=os.cpu_count() or 1)
        assert np.array_equal(rt.trace(torch.tensor(rays, device="cuda"), mode).cpu().numpy(), want)
    rt.close()


def test_trace_binned_with_edge_on_large_and_parallel_triangles():
    """Triangles seen edge-on, larger than the bin limit, parallel to the rays, and exact
    duplicates (ties go to the first) next to the regular surface: same codes as the oracle."""
    ids, abc = ray_surface(10, 12)
    rays = RT.MakeRays(31)
    d = rays[0, 3:]
    rng = np.random.default_rng(5)
    extra = []
    for _ in range(40):  # edge-on: two vertices along the ray direction
        p = rng.uniform([0.5, -0.3, -0.2], [1.3, 0.3, 0.2])
        q = rng.normal(size=3) * 0.05
        extra.append(np.concatenate([p, p + 0.1 * d, p + q]))
    for _ in range(5):  # large
        c = rng.uniform([0.6, -0.2, -0.1], [1.2, 0.2, 0.1])
        extra.append(np.concatenate([c + rng.normal(size=3) * 0.4 for _ in range(3)]))
    extra.append(abc[7].copy())  # duplicate of a surface triangle (later id loses the tie)
    abc2 = np.concatenate([abc, np.array(extra)])
    ids2 = np.concatenate([ids, np.arange(len(extra), dtype=np.int32) + 4 * len(abc) + 100])
    rt = RT.RayTracer(RT.face_cells(ids2, abc2))
    for mode in (RT.SURFACE, RT.ROCHE):
        want = oracle.port_ray_trace(mode, rays, ids2, abc2, nthreads=os.cpu_count() or 1)
        assert np.array_equal(rt.trace(torch.tensor(rays, device="cuda"), mode).cpu().numpy(), want)
    rt.close()


def test_trace_matches_reference_golden_fixture():
    g = np.load(os.path.join(HERE, "golden", "ray.npz"))
    rt = RT.RayTracer(RT.face_cells(g["ids"], g["abc"]))
    rays = torch.tensor(np.ascontiguousarray(g["rays"].reshape(-1, 6)), device="cuda")
    for mode in range(4):
        assert np.array_equal(rt.trace(rays, mode).cpu().numpy(), g["codes"][mode])
    rt.close()


def test_image_and_curve():
    ids, abc = ray_surface(8, 8)
    rays = RT.MakeRays(50)
    rt = RT.RayTracer(RT.face_cells(ids, abc))
    codes = rt.trace(torch.tensor(rays, device="cuda"), RT.INNER)
    rng = np.random.default_rng(4)
    values = rng.uniform(0.5, 2.0, int(ids.max()) // 4 + 1)
    img, curve = RT.RayTracer.image(codes, torch.tensor(values, device="cuda"))
    c = codes.cpu().numpy()
    want = np.select([c == -1, c == -4, c == -2, c == -3], [0.0, 1e-5, 5.0, 10.0],
                     default=values[np.maximum(c, 0) // 4])
    assert np.array_equal(img.cpu().numpy(), want)
    assert curve == pytest.approx(np.sum(want * RT.PIXEL_AREA), rel=1e-13)
    rt.close()


def test_empty_surface_and_invalid_arguments():
    from radrhd_solver_b200 import _lib as L
    rt = RT.RayTracer(RT.face_cells(np.zeros(0, dtype=np.int32), np.zeros((0, 9))))
    rays = torch.tensor(RT.MakeRays(0)[:1000], device="cuda")
    assert torch.all(rt.trace(rays, RT.SURFACE) == RT.NONE)
    codes = torch.empty(1000, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.lib.rrhd_ray_trace(rt._h, rays.data_ptr(), 1000, 4, codes.data_ptr(), s) == L.RRHD_ERR_INVALID
    torch.cuda.synchronize()
    rt.close()
