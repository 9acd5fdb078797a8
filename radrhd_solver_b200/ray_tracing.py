"""Image-plane ray tracing (the reference's ray_tracing module) on the GPU.

Mirrors cuda::ray_tracing::interface (cuda/src/ray_tracing/cuda_ray_interface.cu):
InitDevice(faces) -> RayTracer(face_cells); StartTracing / TracingGrid /
FindInnerIntersection -> RayTracer.trace(rays, mode); ray_tracing::MakeRays(frame)
(solvers/ray_tracing/src/ray_tracing_build_plane.cpp) -> MakeRays(frame); one frame of
MakeIllumAndCurve (ray_tracing_calc_illum.cpp) -> RayTracer.image(codes, values).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

SURFACE, ROCHE, INNER, GRID = 0, 1, 2, 3  # RayTracing, RayTracing_Phl1445, InnerRayTracing, RayTracingGrid
NONE, DISK, SPHERE, LOBE = -1, -2, -3, -4  # e_ray_intersect_code (ray_tracing_const.h)
PIXELS = (600, 300)
PIXEL_AREA = (1.2 / 600) * (0.6 / 300)  # (k_width_plane / k_pixels_width) * (k_height_plane / k_pixels_height)

FACE_CELL = np.dtype([("face_id", "<i4"), ("pad", "<i4"), ("A", "<f8", 3), ("B", "<f8", 3), ("C", "<f8", 3)])


def face_cells(ids, abc) -> np.ndarray:
    """FaceCell records (lib/geometry/include/geo_types.h:77-83, 80 bytes) from ids [n]
    and vertices [n][9] = {A, B, C}."""
    abc = np.asarray(abc, dtype=np.float64).reshape(-1, 9)
    rec = np.zeros(len(abc), dtype=FACE_CELL)
    rec["face_id"] = ids
    rec["A"], rec["B"], rec["C"] = abc[:, 0:3], abc[:, 3:6], abc[:, 6:9]
    return rec


def MakeRays(frame: int) -> np.ndarray:
    """Rays [600 * 300][6] = {orig, direction} of frame `frame`, ray i * 300 + j."""
    rays = np.empty((PIXELS[0] * PIXELS[1], 6))
    L.check(L.lib.rrhd_ray_make_rays(frame, rays.ctypes.data), "rrhd_ray_make_rays")
    return rays


class RayTracer:
    """A triangle surface resident on one GPU."""

    def __init__(self, cells: np.ndarray, device: int = 0):
        cells = np.ascontiguousarray(cells, dtype=FACE_CELL)
        h = C.c_void_p()
        L.check(L.lib.rrhd_ray_surface_create(cells.ctypes.data, len(cells), device, C.byref(h)),
                "rrhd_ray_surface_create")
        self._h = h
        self.n = len(cells)

    def trace(self, rays, mode: int = SURFACE, codes=None, stream=None):
        """Intersection code per ray; rays: CUDA float64 [M, 6]."""
        import torch
        assert rays.is_cuda and rays.dtype == torch.float64 and rays.is_contiguous() and rays.shape[-1] == 6
        M = rays.numel() // 6
        if codes is None:
            codes = torch.empty(M, dtype=torch.int32, device=rays.device)
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        L.check(L.lib.rrhd_ray_trace(self._h, rays.data_ptr(), M, mode, codes.data_ptr(), s), "rrhd_ray_trace")
        return codes

    @staticmethod
    def image(codes, values, cell_size: int = 4, pixel_factor: float = PIXEL_AREA, stream=None):
        """(image [M], curve value) of one frame; values: CUDA float64 per cell."""
        import torch
        M = codes.numel()
        img = torch.empty(M, dtype=torch.float64, device=codes.device)
        curve = torch.empty(1, dtype=torch.float64, device=codes.device)
        bad = torch.zeros(1, dtype=torch.int32, device=codes.device)
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(codes.device).cuda_stream
        L.check(L.lib.rrhd_ray_image(codes.data_ptr(), M, values.data_ptr(), cell_size, pixel_factor,
                                     img.data_ptr(), curve.data_ptr(), bad.data_ptr(), s), "rrhd_ray_image")
        if int(bad.item()):
            raise RuntimeError("rrhd_ray_image: a negative intersection code that is not a known body")
        return img, float(curve.item())

    def close(self):
        if self._h:
            L.lib.rrhd_ray_surface_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
