"""The placer's two objectives as differentiable functions over the C ABI (`gpl_fn_*`).

The reference takes only the forces (gradients) of its objectives: the WA wirelength's in
`update_wirelength_force_wa` + `wl_gradient_pin` (src/nesterov.rs:2325-2430) and the
electrostatic energy's in `density_gradient` (:2434-2449). Here each objective is a
`torch.autograd.Function` whose forward is the engine's value kernel and whose backward is
its hand-written adjoint kernel, both in double on the device, so a caller can put them in an
autograd graph (a loss over cell positions, net weights held fixed):

    W = wirelength(pin_xy, net_start, net_weight, coef_x, coef_y)   # pin_xy: (P, 2) float64 CUDA
    E = DensityEnergy(nx, ny, lx, ly, bin_w, bin_h)(cell_xy, half, scale)
    (W + lam * E).backward()                                        # pin_xy.grad, cell_xy.grad

Both run on the current CUDA stream.
"""
import ctypes as C

import torch

from . import engine

_ready = False


def _lib():
    global _ready
    L = engine.lib()
    if not _ready:
        L.gpl_fn_wa_forward.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_void_p]
        L.gpl_fn_wa_backward.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        L.gpl_fn_density_create.restype = C.c_void_p
        L.gpl_fn_density_create.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p]
        L.gpl_fn_density_eval.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_void_p]
        L.gpl_fn_density_destroy.argtypes = [C.c_void_p]
        _ready = True
    return L


def _stream(t):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _check(t, name, dtype):
    if not (t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise TypeError(f"{name}: a contiguous CUDA {dtype} tensor is required")


class _Wirelength(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pin_xy, net_start, net_weight, coef_x, coef_y):
        _check(pin_xy, "pin_xy", torch.float64)
        _check(net_start, "net_start", torch.int64)
        _check(net_weight, "net_weight", torch.float32)
        v = C.c_double()
        rc = _lib().gpl_fn_wa_forward(net_start.numel() - 1, net_start.data_ptr(), pin_xy.data_ptr(), net_weight.data_ptr(), float(coef_x), float(coef_y), C.byref(v), _stream(pin_xy))
        if rc != 0:
            raise RuntimeError(f"gpl_fn_wa_forward: CUDA error {rc}")
        ctx.save_for_backward(pin_xy, net_start, net_weight)
        ctx.coef = (float(coef_x), float(coef_y))
        return torch.tensor(v.value, dtype=torch.float64, device=pin_xy.device)

    @staticmethod
    def backward(ctx, g):
        pin_xy, net_start, net_weight = ctx.saved_tensors
        grad = torch.zeros_like(pin_xy)
        rc = _lib().gpl_fn_wa_backward(net_start.numel() - 1, net_start.data_ptr(), pin_xy.data_ptr(), net_weight.data_ptr(), ctx.coef[0], ctx.coef[1], float(g), grad.data_ptr(), _stream(pin_xy))
        if rc != 0:
            raise RuntimeError(f"gpl_fn_wa_backward: CUDA error {rc}")
        return grad, None, None, None, None


def wirelength(pin_xy, net_start, net_weight, coef_x, coef_y):
    """The WA wirelength of the nets (pins net-major, net_start of n_nets + 1) at pin_xy."""
    return _Wirelength.apply(pin_xy, net_start, net_weight, coef_x, coef_y)


class _Density(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cell_xy, half, scale, fn):
        for t, n in ((cell_xy, "cell_xy"), (half, "half"), (scale, "scale")):
            _check(t, n, torch.float64)
        e = C.c_double()
        rc = _lib().gpl_fn_density_eval(fn._f, scale.numel(), cell_xy.data_ptr(), half.data_ptr(), scale.data_ptr(), C.byref(e), 0.0, None)
        if rc != 0:
            raise RuntimeError(f"gpl_fn_density_eval: CUDA error {rc}")
        ctx.save_for_backward(cell_xy, half, scale)
        ctx.fn = fn
        return torch.tensor(e.value, dtype=torch.float64, device=cell_xy.device)

    @staticmethod
    def backward(ctx, g):
        cell_xy, half, scale = ctx.saved_tensors
        grad = torch.zeros_like(cell_xy)
        rc = _lib().gpl_fn_density_eval(ctx.fn._f, scale.numel(), cell_xy.data_ptr(), half.data_ptr(), scale.data_ptr(), None, float(g), grad.data_ptr())
        if rc != 0:
            raise RuntimeError(f"gpl_fn_density_eval: CUDA error {rc}")
        return grad, None, None, None


class DensityEnergy:
    """E = 1/2 rho^T G rho over an nx x ny grid of bin_w x bin_h bins from (lx, ly): rho the
    cells' overlap areas (centres cell_xy, half sizes half) times their scales, G the
    reference's DCT Poisson solve. The grid's bases are planned once (on the current stream)."""

    def __init__(self, nx, ny, lx, ly, bin_w, bin_h):
        self._f = _lib().gpl_fn_density_create(nx, ny, lx, ly, bin_w, bin_h, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if not self._f:
            raise RuntimeError("gpl_fn_density_create failed")

    def __call__(self, cell_xy, half, scale):
        return _Density.apply(cell_xy, half, scale, self)

    def close(self):
        if self._f:
            _lib().gpl_fn_density_destroy(self._f)
            self._f = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
