"""The module kernels as PyTorch operators: ``torch.ops.pbemcs.*``.

Importing this module registers three custom operators in the PyTorch dispatcher, each a
thin call into libpbemcs.so on the tensor's current CUDA stream:

    torch.ops.pbemcs.accumulate_rho(x, y, rho, num_p, dx, dy, nx, ny, charge_density)
        ``accumulate_rho`` (Python/physics_engine.py:38-60, 178-185); rho updated in place
    torch.ops.pbemcs.push_particles_boris(x, y, vx, vy, vz, Ex, Ey, Bx, By, Bz,
                                          num_p, dx, dy, nx, ny, dt, q_m)
        ``push_particles_boris`` (:63-144, 188-254); x, y, vx, vy, vz updated in place
    torch.ops.pbemcs.thermal_conduction(T, T_new, mask, nx, ny, Fo_x, Fo_y)
        the Taichi ``thermal_conduction`` kernel (:147-171); T_new written

Arguments keep the reference functions' order and meaning; arrays are contiguous CUDA
tensors (float32, the mask int32).  The operators declare what they mutate, so they can be
used inside code that torch.compile traces or CUDA graphs capture, and they have kernels
for CUDA only: CPU tensors raise instead of falling back.  The same calls without the
dispatcher are ``physics_engine.accumulate_rho`` and friends."""
import torch

from . import _lib

_F32 = torch.float32


def _need(t, name, dtype=_F32):
    if not t.is_cuda:
        raise RuntimeError(f"pbemcs: {name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise RuntimeError(f"pbemcs: {name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise RuntimeError(f"pbemcs: {name} must be contiguous")


def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


@torch.library.custom_op("pbemcs::accumulate_rho", mutates_args=("rho",), device_types="cuda")
def accumulate_rho(x: torch.Tensor, y: torch.Tensor, rho: torch.Tensor, num_p: int, dx: float, dy: float,
                   nx: int, ny: int, charge_density: float) -> None:
    for t, n in ((x, "x"), (y, "y"), (rho, "rho")):
        _need(t, n)
    if rho.numel() < nx * ny or min(x.numel(), y.numel()) < num_p:
        raise RuntimeError("pbemcs: accumulate_rho: arrays smaller than num_p / nx * ny")
    _lib.check(_lib.load().pb_accumulate_rho(x.data_ptr(), y.data_ptr(), rho.data_ptr(), int(num_p), float(dx),
                                             float(dy), int(nx), int(ny), float(charge_density), _stream(rho)),
               "accumulate_rho")


@torch.library.custom_op("pbemcs::push_particles_boris", mutates_args=("x", "y", "vx", "vy", "vz"),
                         device_types="cuda")
def push_particles_boris(x: torch.Tensor, y: torch.Tensor, vx: torch.Tensor, vy: torch.Tensor, vz: torch.Tensor,
                         Ex: torch.Tensor, Ey: torch.Tensor, Bx: torch.Tensor, By: torch.Tensor, Bz: torch.Tensor,
                         num_p: int, dx: float, dy: float, nx: int, ny: int, dt: float, q_m: float) -> None:
    for t, n in ((x, "x"), (y, "y"), (vx, "vx"), (vy, "vy"), (vz, "vz"), (Ex, "Ex"), (Ey, "Ey"), (Bx, "Bx"),
                 (By, "By"), (Bz, "Bz")):
        _need(t, n)
    if min(t.numel() for t in (x, y, vx, vy, vz)) < num_p or min(t.numel() for t in (Ex, Ey, Bx, By, Bz)) < nx * ny:
        raise RuntimeError("pbemcs: push_particles_boris: arrays smaller than num_p / nx * ny")
    _lib.check(_lib.load().pb_push_particles_boris(x.data_ptr(), y.data_ptr(), vx.data_ptr(), vy.data_ptr(),
                                                   vz.data_ptr(), Ex.data_ptr(), Ey.data_ptr(), Bx.data_ptr(),
                                                   By.data_ptr(), Bz.data_ptr(), int(num_p), float(dx), float(dy),
                                                   int(nx), int(ny), float(dt), float(q_m), _stream(x)),
               "push_particles_boris")


@torch.library.custom_op("pbemcs::thermal_conduction", mutates_args=("T_new",), device_types="cuda")
def thermal_conduction(T: torch.Tensor, T_new: torch.Tensor, mask: torch.Tensor, nx: int, ny: int, Fo_x: float,
                       Fo_y: float) -> None:
    _need(T, "T")
    _need(T_new, "T_new")
    _need(mask, "mask", torch.int32)
    if min(T.numel(), T_new.numel(), mask.numel()) < nx * ny:
        raise RuntimeError("pbemcs: thermal_conduction: arrays smaller than nx * ny")
    _lib.check(_lib.load().pb_thermal_conduction(T.data_ptr(), T_new.data_ptr(), mask.data_ptr(), int(nx), int(ny),
                                                 float(Fo_x), float(Fo_y), _stream(T)), "thermal_conduction")


# tracing (torch.compile, meta tensors): the operators return nothing and only mutate
@accumulate_rho.register_fake
def _(x, y, rho, num_p, dx, dy, nx, ny, charge_density):
    return None


@push_particles_boris.register_fake
def _(x, y, vx, vy, vz, Ex, Ey, Bx, By, Bz, num_p, dx, dy, nx, ny, dt, q_m):
    return None


@thermal_conduction.register_fake
def _(T, T_new, mask, nx, ny, Fo_x, Fo_y):
    return None
