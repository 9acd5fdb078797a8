"""The drop-in adapters (adapter/*.cpp), built under the reference's own headers by
`make -C oracle ref`, define the reference's functions with the reference's signatures:
the symbols a maintainer's link resolves against them."""
import os
import shutil
import subprocess

import pytest

import oracle

WANT = {
    "adapter_hydro_5_3": ["rhllc::Hllc3dStab(double, grid_t&)"],
    "adapter_rad": [
        "cuda::interface::separate_device::InitDevice(grid_directions_t const&, grid_t&)",
        "cuda::interface::separate_device::ClearDevice()",
        "cuda::interface::separate_device::ClearHost(grid_t&)",
        "cuda::interface::separate_device::CalculateIntScatteringAsync(grid_directions_t const&, grid_t&, long, long, "
        "cuda::e_cuda_stream_id_t)",
        "cuda::interface::separate_device::CalculateAllParamAsync(int, int, grid_directions_t const&, grid_t&, "
        "cuda::e_cuda_stream_id_t)",
        "cuda::interface::SetStreams()", "cuda::interface::CudaWait()",
        "cuda::interface::CudaSyncStream(cuda::e_cuda_stream_id_t)",
        "cuda::interface::CudaSendIllumAsync(long, long, double const*)",
    ],
    "adapter_rad_spectrum": [
        "cuda::interface::separate_device::SendVelocity(grid_t const&)",
        "cuda::interface::separate_device::CalculateSpectrumIntScattering(grid_directions_t const&, grid_t&, long, long, "
        "cuda::e_cuda_stream_id_t)",
        "cuda::interface::separate_device::CalculateFullSpectrumIntScattering(grid_directions_t const&, grid_t&, long, "
        "long, cuda::e_cuda_stream_id_t)",
    ],
    "adapter_ray": [
        "cuda::ray_tracing::interface::InitDevice(std::vector<FaceCell, std::allocator<FaceCell> > const&, "
        "std::vector<Ray_t, std::allocator<Ray_t> > const&)",
        "cuda::ray_tracing::interface::ClearDevice()",
        "cuda::ray_tracing::interface::StartTracing(std::vector<Ray_t, std::allocator<Ray_t> > const&, "
        "std::vector<int, std::allocator<int> >&)",
    ],
}


@pytest.mark.parametrize("variant", sorted(WANT))
def test_adapter_defines_the_reference_functions(variant):
    if not oracle.have_ref(variant):
        pytest.skip(f"{variant} not built (make -C oracle ref)")
    if shutil.which("nm") is None:
        pytest.skip("nm not available")
    path = os.path.join(oracle.loader.REF_DIR, f"librrhd_ref_{variant}.so")
    out = subprocess.run(["nm", "-DC", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    for sym in WANT[variant]:
        assert sym in out, f"{variant} does not define {sym}"
