"""Helpers for the GPU tests: run the library through its C-ABI on device buffers."""
import numpy as np


def run_device(plan, x_np, inverse=False):
    """Copy x to the GPU (torch memory), run the plan through fmmfft_execute, copy back."""
    import torch
    dt = torch.complex128 if plan.precision == "f64" else torch.complex64
    x = torch.from_numpy(np.ascontiguousarray(x_np)).to(dt).cuda()
    y = torch.empty_like(x)
    plan.execute_ptr(x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream, inverse)
    torch.cuda.synchronize()
    return y.cpu().numpy().astype(np.complex128)
