"""ctypes front end of the CPU oracle (liboracle.so, built from lbm_oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py use this module, and only as the checker or the
timed CPU baseline; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
# the same source built for speed (-O3, FMA contraction, AVX2): only the timed
# CPU baseline uses it; parity always uses LIB
LIB_FAST = HERE / "liboracle_fast.so"

_lib = None
_lib_fast = None
_P = C.c_void_p


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib(fast: bool = False) -> C.CDLL:
    global _lib, _lib_fast
    if fast:
        if _lib_fast is None:
            if not LIB_FAST.exists():
                build()
            _lib_fast = _bind(C.CDLL(str(LIB_FAST)))
        return _lib_fast
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = _bind(C.CDLL(str(LIB)))
    return _lib


def _bind(L: C.CDLL) -> C.CDLL:
    sigs = {
        "oracle_set_threads": (None, [C.c_int]),
        "oracle_max_threads": (C.c_int, []),
        "oracle_tables": (None, [_P, _P, _P]),
        "oracle_feq_f64": (None, [C.c_double] * 4 + [_P]),
        "oracle_feq_f32": (None, [C.c_float] * 4 + [_P]),
        "oracle_round_f16": (C.c_float, [C.c_float, C.c_int]),
        "oracle_classify": (None, [C.c_int, C.c_int, C.c_int, _P, _P, _P]),
        "oracle_ref_init": (None, [_P, _P, _P, _P, C.c_float, _P, _P, _P, _P]),
        "oracle_ref_step": (None, [_P, _P, _P, _P, _P, _P, C.c_int]),
        "oracle_ref_collided": (None, [_P, _P, _P, _P, _P, _P]),
        "oracle_ext_init_f64": (None, [_P] * 6),
        "oracle_ext_init_f32": (None, [_P] * 6),
        "oracle_ext_step_f64": (None, [_P, _P, _P, _P, C.c_int, _P, _P]),
        "oracle_ext_step_f32": (None, [_P, _P, _P, _P, C.c_int, _P, _P]),
        "oracle_voxelize_naca": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                           C.c_float, C.c_float, _P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def _p(a) -> int | None:
    return None if a is None else a.ctypes.data


def set_threads(n: int) -> None:
    lib().oracle_set_threads(n)
    lib(fast=True).oracle_set_threads(n)


def max_threads() -> int:
    return lib().oracle_max_threads()


def tables():
    c = np.zeros((19, 3), np.int32)
    w = np.zeros(19, np.float64)
    o = np.zeros(19, np.int32)
    lib().oracle_tables(_p(c), _p(w), _p(o))
    return c, w, o


def feq_f64(rho, ux, uy, uz) -> np.ndarray:
    out = np.zeros(19, np.float64)
    lib().oracle_feq_f64(rho, ux, uy, uz, _p(out))
    return out


def feq_f32(rho, ux, uy, uz) -> np.ndarray:
    out = np.zeros(19, np.float32)
    lib().oracle_feq_f32(rho, ux, uy, uz, _p(out))
    return out


def round_f16(v: float, mode: int = 1) -> float:
    return lib().oracle_round_f16(v, mode)


def classify(mask: np.ndarray, shape, periodic=(0, 0, 0)) -> np.ndarray:
    nx, ny, nz = shape
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    per = np.array(periodic, np.int32)
    out = np.zeros(nx * ny * nz, np.uint32)
    lib().oracle_classify(nx, ny, nz, _p(per), _p(m), _p(out))
    return out


def voxelize_naca(designation, nx, ny, nz, chord_frac=0.25, center_x_frac=0.25, aoa_deg=0.0):
    m = np.zeros(nx * ny * nz, np.uint8)
    lib().oracle_voxelize_naca(designation.encode(), nx, ny, nz, chord_frac, center_x_frac, aoa_deg, _p(m))
    return m


class RefState:
    """The reference's state between substeps: ping populations float[19][N]
    and the rho / u moment images (u kept unrounded; the collide rounds)."""

    def __init__(self, shape, tau=0.6, u_inf=(0.0, 0.0, 0.0), rho0=1.0, inlet_outlet=1,
                 free_slip=1, u_round=1, mask=None):
        self.shape = tuple(shape)
        nx, ny, nz = self.shape
        self.n = nx * ny * nz
        self.ip = np.array([nx, ny, nz, inlet_outlet, free_slip, u_round], np.int32)
        self.fp = np.array([tau, u_inf[0], u_inf[1], u_inf[2], rho0], np.float32)
        self.mask = np.zeros(self.n, np.uint8) if mask is None else np.ascontiguousarray(mask, np.uint8).reshape(-1)
        self.f = np.zeros((19, self.n), np.float32)
        self.rho = np.zeros(self.n, np.float32)
        self.u = np.zeros((3, self.n), np.float32)

    def init(self, rho0=1.0, u0=(0.0, 0.0, 0.0), rho=None, u=None):
        """u: float[3][N] planes or None."""
        u0a = np.array(u0, np.float32)
        r = None if rho is None else np.ascontiguousarray(rho, np.float32).reshape(-1)
        uu = None if u is None else np.ascontiguousarray(u, np.float32).reshape(3, -1)
        lib().oracle_ref_init(_p(self.ip), _p(self.fp), _p(r), _p(uu), rho0, _p(u0a),
                              _p(self.f), _p(self.rho), _p(self.u))

    def set_params(self, tau=None, u_inf=None):
        """A uniform change between frames (src/main.cpp:1523-1537): the next
        collide uses the new tau, the next boundary pass the new u_inf."""
        if tau is not None:
            self.fp[0] = tau
        if u_inf is not None:
            self.fp[1:4] = u_inf

    def step(self, n=1):
        lib().oracle_ref_step(_p(self.ip), _p(self.fp), _p(self.mask), _p(self.f), _p(self.rho),
                              _p(self.u), n)

    def collided(self) -> np.ndarray:
        """Post-collision populations of the next step (what the fused GPU
        kernel keeps between launches)."""
        out = np.zeros_like(self.f)
        lib().oracle_ref_collided(_p(self.ip), _p(self.fp), _p(self.f), _p(self.rho), _p(self.u), _p(out))
        return out


def _ext_dp(tau, trt_magic, smag_cs, accel, wall, net, open_rho=(0.0, 0.0)):
    """Double parameters of ExtStep (ext_step.h make_ext): tau, Lambda, Cs,
    accel[3], wall[6][3], open_rho[2], has_net, then the network (its weights
    as the kernels use them, rounded to bf16) if one is given."""
    parts = [[tau, trt_magic, smag_cs], np.asarray(accel, np.float64), np.asarray(wall, np.float64).reshape(-1),
             np.asarray(open_rho, np.float64)]
    if net is None:
        parts.append([0.0])
    else:
        from .closure_oracle import kernel_net
        parts += [[1.0], kernel_net(net).astype(np.float64)]
    return np.ascontiguousarray(np.concatenate(parts), np.float64)


def _set_ext_params(dp, tau, accel, wall, smag_cs):
    if tau is not None:
        dp[0] = tau
    if smag_cs is not None:
        dp[2] = smag_cs
    if accel is not None:
        dp[3:6] = accel
    if wall is not None:
        dp[6:24] = np.asarray(wall, np.float64).reshape(-1)


class ExtState:
    """Textbook stream-collide state: post-collision populations float[19][N]."""

    def __init__(self, shape, periodic=(0, 0, 0), tau=0.6, collision=0, trt_magic=3.0 / 16.0,
                 smag_cs=0.0, accel=(0.0, 0.0, 0.0), wall=None, mask=None, dtype=np.float64,
                 net=None, open_x=(0, 0), open_rho=(0.0, 0.0), fast=False):
        """fast: run on the speed build (the timed CPU baseline); results may
        differ from the checker build in the last place (FMA contraction)."""
        self.fast = fast
        self.shape = tuple(shape)
        nx, ny, nz = self.shape
        self.n = nx * ny * nz
        self.dtype = np.dtype(dtype)
        self.ip = np.array([nx, ny, nz, *periodic, collision, *open_x], np.int32)
        w = np.zeros((6, 3)) if wall is None else np.asarray(wall, np.float64).reshape(6, 3)
        self.dp = _ext_dp(tau, trt_magic, smag_cs, accel, w, net, open_rho)
        self.mask = np.zeros(self.n, np.uint8) if mask is None else np.ascontiguousarray(mask, np.uint8).reshape(-1)
        self.f = np.zeros((19, self.n), self.dtype)
        self.rho = np.zeros(self.n, self.dtype)
        self.u = np.zeros((3, self.n), self.dtype)

    def init(self, rho, u):
        r = np.ascontiguousarray(np.broadcast_to(rho, (self.n,)), self.dtype)
        uu = np.ascontiguousarray(np.asarray(u, self.dtype).reshape(3, -1) * np.ones((3, self.n)), self.dtype)
        L = lib(self.fast)
        fn = L.oracle_ext_init_f64 if self.dtype == np.float64 else L.oracle_ext_init_f32
        fn(_p(self.ip), _p(self.dp), _p(self.mask), _p(r), _p(uu), _p(self.f))
        self.rho[:] = np.where(self.mask == 1, 0, r)
        self.u[:] = np.where(self.mask == 1, 0, uu)

    def set_params(self, tau=None, accel=None, wall=None, smag_cs=None):
        """New parameters from the next step on (layout of _ext_dp)."""
        _set_ext_params(self.dp, tau, accel, wall, smag_cs)

    def step(self, n=1):
        L = lib(self.fast)
        fn = L.oracle_ext_step_f64 if self.dtype == np.float64 else L.oracle_ext_step_f32
        fn(_p(self.ip), _p(self.dp), _p(self.mask), _p(self.f), n, _p(self.rho), _p(self.u))


LIB_GPU = HERE / "liboracle_gpu.so"
_lib_gpu = None


def lib_gpu() -> C.CDLL:
    global _lib_gpu
    if _lib_gpu is None:
        if not LIB_GPU.exists():
            build()
        L = C.CDLL(str(LIB_GPU))
        L.oracle_gpu_ext_init_f64.restype = C.c_int
        L.oracle_gpu_ext_init_f64.argtypes = [_P] * 6
        L.oracle_gpu_ext_step_f64.restype = C.c_int
        L.oracle_gpu_ext_step_f64.argtypes = [_P, _P, _P, _P, _P, C.c_int, _P, _P]
        _lib_gpu = L
    return _lib_gpu


class ExtStateGPU:
    """FP64 ExtStep on the current CUDA device (same node update as ExtState,
    bit for bit); device memory through torch.  For full-size FP64 runs."""

    def __init__(self, shape, periodic=(0, 0, 0), tau=0.6, collision=0, trt_magic=3.0 / 16.0,
                 smag_cs=0.0, accel=(0.0, 0.0, 0.0), wall=None, mask=None, net=None, open_x=(0, 0),
                 open_rho=(0.0, 0.0)):
        import torch
        self.torch = torch
        self.shape = tuple(shape)
        nx, ny, nz = self.shape
        self.n = nx * ny * nz
        self.ip = np.array([nx, ny, nz, *periodic, collision, *open_x], np.int32)
        w = np.zeros((6, 3)) if wall is None else np.asarray(wall, np.float64).reshape(6, 3)
        self.dp = _ext_dp(tau, trt_magic, smag_cs, accel, w, net, open_rho)
        m = np.zeros(self.n, np.uint8) if mask is None else np.ascontiguousarray(mask, np.uint8).reshape(-1)
        dev = torch.device("cuda")
        self.mask = torch.from_numpy(m).to(dev)
        self.f = torch.zeros(19 * self.n, dtype=torch.float64, device=dev)
        self.tmp = torch.zeros_like(self.f)
        self.rho = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self.u = torch.zeros(3 * self.n, dtype=torch.float64, device=dev)

    def init(self, rho, u):
        t = self.torch
        r = t.from_numpy(np.array(np.broadcast_to(rho, (self.n,)), np.float64)).cuda()  # a writable copy
        uu = t.from_numpy(np.ascontiguousarray(np.asarray(u, np.float64).reshape(3, -1) * np.ones((3, self.n)))).cuda()
        t.cuda.synchronize()
        rc = lib_gpu().oracle_gpu_ext_init_f64(self.ip.ctypes.data, self.dp.ctypes.data, self.mask.data_ptr(),
                                               r.data_ptr(), uu.data_ptr(), self.f.data_ptr())
        assert rc == 0, rc
        self.rho.copy_(r)
        self.u.copy_(uu.reshape(-1))
        solid = self.mask == 1
        self.rho[solid] = 0
        self.u.view(3, -1)[:, solid] = 0

    def set_params(self, tau=None, accel=None, wall=None, smag_cs=None):
        _set_ext_params(self.dp, tau, accel, wall, smag_cs)

    def step(self, n=1):
        self.torch.cuda.synchronize()
        rc = lib_gpu().oracle_gpu_ext_step_f64(self.ip.ctypes.data, self.dp.ctypes.data, self.mask.data_ptr(),
                                               self.f.data_ptr(), self.tmp.data_ptr(), n,
                                               self.rho.data_ptr(), self.u.data_ptr())
        assert rc == 0, rc

    def moments(self):
        return self.rho.cpu().numpy(), self.u.view(3, -1).cpu().numpy()
