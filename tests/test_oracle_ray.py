"""The image-plane ray-tracing oracle (C restatement of cuda/src/ray_tracing/cuda_ray_calc.cu,
cuda_ray_geo_intersect.cu and ray_tracing_build_plane.cpp's MakeRays) pinned bit for bit to
the reference's own sources compiled for the host (oracle/_ref, where built) and to the
golden fixture tests/golden/ray.npz made from them; the library's host-side
rrhd_ray_make_rays against the same."""
import os

import numpy as np
import pytest

import oracle
from cases import ray_surface
from oracle import loader as Ld

HERE = os.path.dirname(os.path.abspath(__file__))
have_ref = pytest.mark.skipif(not oracle.have_ref("ray"), reason="reference ray tracing not built (make -C oracle ref)")


def test_port_matches_golden_fixture():
    g = np.load(os.path.join(HERE, "golden", "ray.npz"))
    for f, R in zip(g["frames"], g["rays"]):
        assert np.array_equal(oracle.port_ray_make_rays(int(f))[g["sample"]], R)
    for mode in range(4):
        assert np.array_equal(oracle.port_ray_trace(mode, g["rays"].reshape(-1, 6), g["ids"], g["abc"], nthreads=4),
                              g["codes"][mode])


def test_library_make_rays_matches_golden_fixture():
    from radrhd_solver_b200 import ray_tracing
    g = np.load(os.path.join(HERE, "golden", "ray.npz"))
    for f, R in zip(g["frames"], g["rays"]):
        assert np.array_equal(ray_tracing.MakeRays(int(f))[g["sample"]], R)


@have_ref
@pytest.mark.parametrize("frame", [0, 23, 60, 101])
def test_make_rays_matches_reference(frame):
    from radrhd_solver_b200 import ray_tracing
    R = oracle.ref_ray_make_rays(frame)
    assert np.array_equal(oracle.port_ray_make_rays(frame), R)
    assert np.array_equal(ray_tracing.MakeRays(frame), R)


@have_ref
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_trace_matches_reference(mode):
    ids, abc = ray_surface(6, 8)
    rays = oracle.port_ray_make_rays(7)[::41]
    want = oracle.ref_ray(mode, rays, ids, abc)
    assert np.array_equal(oracle.port_ray_trace(mode, rays, ids, abc, nthreads=4), want)
    assert len(np.unique(want)) > 20


@have_ref
def test_unit_functions_match_reference():
    rng = np.random.default_rng(2)
    ids, abc = ray_surface(4, 6)
    for i in range(3000):
        r = np.concatenate([rng.uniform(-1, 2, 3), rng.normal(size=3)])
        assert Ld.port_ray_triangle(r, abc[i % len(abc)]) == Ld.ref_ray_triangle(r, abc[i % len(abc)])
        assert Ld.port_ray_roche(r) == Ld.ref_ray_roche(r)


def test_nearest_hit_takes_first_of_equal_distances():
    """Two copies of a triangle under different ids: the first in input order wins."""
    abc = np.array([[0.0, -1, -1, 0, 1, -1, 0, 0, 1]] * 2)
    rays = np.array([[-1.0, 0, 0, 1, 0, 0], [-1.0, 5, 0, 1, 0, 0]])
    out = oracle.port_ray_trace(0, rays, np.array([7, 3], dtype=np.int32), abc)
    assert list(out) == [7, -1]
