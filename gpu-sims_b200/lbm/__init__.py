"""Python host layer over the C ABI of liblbm_b200.so (include/lbm.h).

It mirrors the reference sim host (volumetric-grid/lattice-boltzmann/src/
main.cpp): the tier and preset tables (:103-135), apply_preset (:1167-1211),
the substep chain (:1554-1591) and the moment readback (:1288-1314).  All
compute goes through the CUDA library; there is no CPU fallback: if the
library is missing, importing a Lattice raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("LBM_B200_LIB", _HERE / "liblbm_b200.so"))

# status codes (include/lbm.h)
OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_NO_DEVICE = -3
ERR_OUT_OF_MEMORY = -4
ERR_STATE = -5
ERR_UNSUPPORTED = -6
ERR_TIMEOUT = -7
ERR_NONFINITE = -8
ERR_IO = -9

MODE_REFERENCE, MODE_PHYSICS = 0, 1
PREC_F32, PREC_F16S, PREC_BF16S = 0, 1, 2
COLL_BGK, COLL_TRT = 0, 1
UROUND_NONE, UROUND_RTE, UROUND_RTZ = 0, 1, 2
U_F32X3, U_F16X4, U_F32X4 = 0, 1, 2
FACE_XM, FACE_XP, FACE_YM, FACE_YP, FACE_ZM, FACE_ZP = range(6)
OPEN_NONE, OPEN_VELOCITY, OPEN_PRESSURE = 0, 1, 2

ERR_NAMES = {OK: "OK", ERR_INVALID_ARG: "INVALID_ARG", ERR_CUDA: "CUDA", ERR_NO_DEVICE: "NO_DEVICE",
             ERR_OUT_OF_MEMORY: "OUT_OF_MEMORY", ERR_STATE: "STATE", ERR_UNSUPPORTED: "UNSUPPORTED",
             ERR_TIMEOUT: "TIMEOUT", ERR_NONFINITE: "NONFINITE", ERR_IO: "IO"}


class LbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Desc(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("mode", C.c_int32), ("precision", C.c_int32), ("collision", C.c_int32),
        ("periodic", C.c_int32 * 3),
        ("tau", C.c_float), ("trt_magic", C.c_float), ("smagorinsky_cs", C.c_float),
        ("body_accel", C.c_float * 3),
        ("wall_velocity", (C.c_float * 3) * 6),
        ("u_inf", C.c_float * 3), ("rho0", C.c_float),
        ("ref_inlet_outlet", C.c_int32), ("ref_free_slip", C.c_int32), ("ref_u_round", C.c_int32),
        ("open_x", C.c_int32 * 2), ("open_rho", C.c_float * 2),
    ]


class Info(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("mode", C.c_int32), ("precision", C.c_int32),
        ("iteration", C.c_uint64), ("device_bytes", C.c_uint64),
        ("bytes_per_node", C.c_double), ("layout", C.c_int32), ("device", C.c_int32),
    ]


class Params(C.Structure):
    """lbm_params: solver parameters changeable between steps."""
    _fields_ = [
        ("struct_size", C.c_uint32), ("tau", C.c_float), ("u_inf", C.c_float * 3),
        ("body_accel", C.c_float * 3), ("wall_velocity", (C.c_float * 3) * 6),
        ("smagorinsky_cs", C.c_float), ("trt_magic", C.c_float), ("open_rho", C.c_float * 2),
    ]


class BatchSchedule(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("rows_per_block", C.c_int32), ("z_per_thread", C.c_int32), ("persistent", C.c_int32),
        ("spin_limit_cycles", C.c_int64), ("test_missing_blocks", C.c_int32),
    ]


class BatchInfo(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("domains", C.c_int32), ("total_nodes", C.c_uint64),
        ("tiles", C.c_uint32), ("grid", C.c_int32), ("iteration", C.c_uint64),
        ("device_bytes", C.c_uint64), ("bytes_per_node", C.c_double),
    ]


class CaptureInfo(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("frame", C.c_uint32), ("iteration", C.c_uint64), ("has_populations", C.c_int32),
        ("mask_frame_invariant", C.c_int32),
    ]


VDB_F32 = 1


def vdb_write_vec3(path: str, xyz: np.ndarray, shape, voxel_size: float = 1.0, origin=None,
                   grid_name: str | None = None) -> None:
    """Writes a dense vec3 grid (xyz float[N][3], x-fastest) as an OpenVDB
    file (lbm_vdb_write_vec3)."""
    a = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    nx, ny, nz = shape
    if a.shape[0] != nx * ny * nz:
        raise LbmError(ERR_INVALID_ARG, "xyz must hold Nx*Ny*Nz vectors")
    org = None if origin is None else (C.c_float * 3)(*origin)
    rc = load().lbm_vdb_write_vec3(str(path).encode(), _ptr(a), nx, ny, nz, voxel_size, org,
                                   None if grid_name is None else grid_name.encode())
    if rc != OK:
        raise LbmError(rc, load().lbm_vdb_last_error().decode())


CAPTURE_LOAD_MASK = 1
CAPTURE_MOMENTS_ONLY = 2


class VelmagParams(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("inv_view_proj", C.c_float * 16), ("camera_pos", C.c_float * 3),
        ("volume_min", C.c_float * 3), ("volume_max", C.c_float * 3), ("steps", C.c_int32),
        ("absorption", C.c_float), ("velmag_min", C.c_float), ("velmag_max", C.c_float),
        ("exposure", C.c_float), ("round_f16", C.c_int32),
    ]


class Adam(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("lr", C.c_float), ("beta1", C.c_float),
        ("beta2", C.c_float), ("eps", C.c_float), ("weight_decay", C.c_float),
    ]


# include/lbm_closure.h
CLOSURE_INPUTS = 9
CLOSURE_HIDDEN = 32
CLOSURE_PARAMS = 1409
CLOSURE_FLOATS = 1427

# Every symbol include/lbm.h and include/lbm_closure.h declare, with its
# ctypes signature.
_P = C.c_void_p
_I32, _I64, _U64, _F = C.c_int32, C.c_int64, C.c_uint64, C.c_float
_SIGS = {
    "lbm_desc_default": (C.c_int, [C.POINTER(Desc)]),
    "lbm_create": (C.c_int, [C.POINTER(Desc), C.POINTER(_P)]),
    "lbm_destroy": (C.c_int, [_P]),
    "lbm_set_stream": (C.c_int, [_P, _P]),
    "lbm_set_flags": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_conservation_async": (C.c_int, [_P, _P]),
    "lbm_set_flags_naca": (C.c_int, [_P, C.c_char_p, C.c_float, C.c_float, C.c_float]),
    "lbm_read_classification": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_init_equilibrium": (C.c_int, [_P, C.c_float, C.POINTER(C.c_float)]),
    "lbm_init_from_moments": (C.c_int, [_P, _P, _P, C.c_int]),
    "lbm_step": (C.c_int, [_P, C.c_int]),
    "lbm_sync": (C.c_int, [_P]),
    "lbm_read_moments": (C.c_int, [_P, _P, _P, C.c_int]),
    "lbm_device_moments": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
    "lbm_conservation": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "lbm_conservation_noalloc": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_double), _P]),
    "lbm_read_populations": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_write_populations": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_get_info": (C.c_int, [_P, C.POINTER(Info)]),
    "lbm_last_error": (C.c_char_p, [_P]),
    "lbm_lattice_tables": (C.c_int, [_P, _P, _P]),
    "lbm_voxelize_naca": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                    C.c_float, C.c_float, _P, C.c_size_t]),
    "lbm_voxelize_naca_device": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                           C.c_float, C.c_float, _P, C.c_size_t, _P]),
    "lbm_half_to_float": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_build_info": (C.c_char_p, []),
    "lbm_batch_schedule_default": (C.c_int, [C.POINTER(BatchSchedule)]),
    "lbm_batch_create": (C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    "lbm_batch_destroy": (C.c_int, [_P]),
    "lbm_batch_set_stream": (C.c_int, [_P, _P]),
    "lbm_batch_set_flags": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "lbm_batch_init_equilibrium": (C.c_int, [_P, C.c_int, C.c_float, C.POINTER(C.c_float)]),
    "lbm_batch_init_from_moments": (C.c_int, [_P, C.c_int, _P, _P, C.c_int]),
    "lbm_batch_step": (C.c_int, [_P, C.c_int]),
    "lbm_batch_sync": (C.c_int, [_P]),
    "lbm_batch_read_moments": (C.c_int, [_P, C.c_int, _P, _P, C.c_int]),
    "lbm_batch_read_populations": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "lbm_batch_set_schedule": (C.c_int, [_P, C.POINTER(BatchSchedule)]),
    "lbm_batch_get_schedule": (C.c_int, [_P, C.POINTER(BatchSchedule)]),
    "lbm_batch_autotune": (C.c_int, [_P, C.c_int, C.POINTER(BatchSchedule)]),
    "lbm_batch_get_info": (C.c_int, [_P, C.POINTER(BatchInfo)]),
    "lbm_batch_last_error": (C.c_char_p, [_P]),
    "lbm_read_mask": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_set_step_variant": (C.c_int, [_P, C.c_int]),
    "lbm_read_populations_shifted": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_write_populations_shifted": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_get_desc": (C.c_int, [_P, C.POINTER(Desc)]),
    "lbm_get_params": (C.c_int, [_P, C.POINTER(Params)]),
    "lbm_set_params": (C.c_int, [_P, C.POINTER(Params)]),
    "lbm_set_iteration": (C.c_int, [_P, _U64]),
    "lbm_capture_write": (C.c_int, [C.c_char_p, C.c_uint32, C.c_char_p, _I32, _I32, _I32, _P, _P, _P, _P]),
    "lbm_capture_read": (C.c_int, [C.c_char_p, C.POINTER(CaptureInfo), _P, _P, _P, _P]),
    "lbm_capture_latest": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t]),
    "lbm_capture_save": (C.c_int, [_P, C.c_char_p, C.c_uint32, C.c_char_p, C.c_int]),
    "lbm_capture_load": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "lbm_capture_last_error": (C.c_char_p, []),
    "lbm_streamline_advect": (C.c_int, [_P, _I32, _I32, _I32, _P, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.c_uint32, _F, C.c_uint32, _I32, _P]),
    "lbm_streamline_seed": (C.c_int, [_P, C.c_uint32, C.c_uint32, _I32, _I32, _I32, C.c_uint32, C.c_uint32]),
    "lbm_velmag_params_default": (C.c_int, [C.POINTER(VelmagParams)]),
    "lbm_render_velmag": (C.c_int, [_P, _I32, _I32, _I32, C.POINTER(VelmagParams), _I32, _I32, _P, _P]),
    "lbm_colormap_lut": (C.c_int, [_P]),
    "lbm_jitter_lut": (C.c_int, [_P]),
    "lbm_set_closure": (C.c_int, [_P, _P]),
    "lbm_set_closure_wait_limit": (C.c_int, [_P, C.c_int32]),
    "lbm_box_filter": (C.c_int, [_P, _P, _I32, _I32, _I32, _I32, _P, _P]),
    "lbm_closure_samples": (C.c_int, [_P, _I32, _I32, _I32, _F, _F, _U64, _I64, _P, _P, _P, _P]),
    "lbm_closure_predict": (C.c_int, [_P, _P, _I64, _P, _P]),
    "lbm_adam_default": (C.c_int, [C.POINTER(Adam)]),
    "lbm_trainer_create": (C.c_int, [_P, C.POINTER(Adam), C.POINTER(_P)]),
    "lbm_trainer_destroy": (C.c_int, [_P]),
    "lbm_trainer_set_stream": (C.c_int, [_P, _P]),
    "lbm_trainer_grad": (C.c_int, [_P, _P, _P, _P, _I64, _F, _P, C.POINTER(C.c_double)]),
    "lbm_trainer_adam_step": (C.c_int, [_P]),
    "lbm_trainer_fit": (C.c_int, [_P, _P, _P, _P, _I64, _I32, _I32, _U64, _P]),
    "lbm_trainer_get_net": (C.c_int, [_P, _P]),
    "lbm_trainer_last_error": (C.c_char_p, [_P]),
    "lbm_round_bf16": (C.c_int, [_P, _P, C.c_size_t]),
    "lbm_vdb_write_vec3": (C.c_int, [C.c_char_p, _P, _I32, _I32, _I32, _F, _P, C.c_char_p]),
    "lbm_vdb_export": (C.c_int, [_P, C.c_char_p, C.c_uint32, C.c_int]),
    "lbm_vdb_last_error": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise LbmError(ERR_STATE, f"{LIB_PATH} is missing: build it with gpu-sims_b200/build.py")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _check(rc: int, ctx=None) -> None:
    if rc != OK:
        msg = load().lbm_last_error(ctx).decode()
        raise LbmError(rc, msg)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def build_info() -> str:
    return load().lbm_build_info().decode()


def lattice_tables():
    """(c[19,3] int32, w[19] float32, opp[19] int32) in the reference order."""
    c = np.zeros((19, 3), np.int32)
    w = np.zeros(19, np.float32)
    o = np.zeros(19, np.int32)
    _check(load().lbm_lattice_tables(_ptr(c), _ptr(w), _ptr(o)))
    return c, w, o


def voxelize_naca(designation: str, nx: int, ny: int, nz: int, chord_frac: float = 0.25,
                  center_x_frac: float = 0.25, angle_of_attack_deg: float = 0.0) -> np.ndarray:
    """Obstacle mask (uint8, x-fastest flat array) of a NACA 4-digit airfoil."""
    m = np.zeros(nx * ny * nz, np.uint8)
    _check(load().lbm_voxelize_naca(designation.encode(), nx, ny, nz, chord_frac, center_x_frac,
                                    angle_of_attack_deg, _ptr(m), m.size))
    return m


def voxelize_naca_device(designation: str, nx: int, ny: int, nz: int, d_mask: int, n: int,
                         chord_frac: float = 0.25, center_x_frac: float = 0.25,
                         angle_of_attack_deg: float = 0.0, stream: int = 0) -> None:
    """The mask of voxelize_naca written on the device into d_mask (a device
    pointer to n = nx*ny*nz bytes) on `stream`; asynchronous."""
    _check(load().lbm_voxelize_naca_device(designation.encode(), nx, ny, nz, chord_frac, center_x_frac,
                                           angle_of_attack_deg, C.c_void_p(d_mask), n,
                                           C.c_void_p(stream or None)))


def half_to_float(h: np.ndarray) -> np.ndarray:
    h = np.ascontiguousarray(h, dtype=np.uint16)
    out = np.empty(h.shape, np.float32)
    _check(load().lbm_half_to_float(_ptr(h), _ptr(out), h.size))
    return out


def default_desc(**kw) -> Desc:
    d = Desc()
    _check(load().lbm_desc_default(C.byref(d)))
    for k, v in kw.items():
        if k in ("periodic", "body_accel", "u_inf", "open_x", "open_rho"):
            arr = getattr(d, k)
            for i, x in enumerate(v):
                arr[i] = x
        elif k == "wall_velocity":
            for f, vec in enumerate(v):
                for a, x in enumerate(vec):
                    d.wall_velocity[f][a] = x
        else:
            setattr(d, k, v)
    return d


class Lattice:
    """One D3Q19 domain on the current CUDA device (wraps an lbm_ctx)."""

    def __init__(self, desc: Desc | None = None, **kw):
        lib = load()
        self.desc = desc if desc is not None else default_desc(**kw)
        h = _P()
        _check(lib.lbm_create(C.byref(self.desc), C.byref(h)))
        self._h = h
        self.shape = (self.desc.nx, self.desc.ny, self.desc.nz)
        self.n = self.desc.nx * self.desc.ny * self.desc.nz

    # context lifetime -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            load().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc: int) -> None:
        _check(rc, self._h)

    # API ---------------------------------------------------------------------
    def set_stream(self, stream_ptr: int | None) -> None:
        self._c(load().lbm_set_stream(self._h, stream_ptr))

    def set_flags(self, mask: np.ndarray) -> None:
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        self._c(load().lbm_set_flags(self._h, _ptr(m), m.size))

    def set_flags_naca(self, designation: str, chord_frac: float = 0.25, center_x_frac: float = 0.25,
                       angle_of_attack_deg: float = 0.0) -> None:
        """set_flags(voxelize_naca(...)) with the mask made on the device."""
        self._c(load().lbm_set_flags_naca(self._h, designation.encode(), chord_frac, center_x_frac,
                                          angle_of_attack_deg))

    def read_populations_shifted(self) -> np.ndarray:
        g = np.empty((19, self.n), np.float32)
        self._c(load().lbm_read_populations_shifted(self._h, _ptr(g), g.size))
        return g

    def write_populations_shifted(self, g: np.ndarray) -> None:
        a = np.ascontiguousarray(g, dtype=np.float32)
        self._c(load().lbm_write_populations_shifted(self._h, _ptr(a), a.size))

    def params(self) -> Params:
        p = Params()
        p.struct_size = C.sizeof(Params)
        self._c(load().lbm_get_params(self._h, C.byref(p)))
        return p

    def set_params(self, **kw) -> None:
        """Changes solver parameters between steps (lbm_set_params), e.g.
        set_params(tau=0.7, u_inf=(0.03, 0.0, 0.0)); unnamed fields keep their
        current values."""
        p = self.params()
        for k, v in kw.items():
            if k in ("u_inf", "body_accel", "open_rho"):
                arr = getattr(p, k)
                for i, x in enumerate(v):
                    arr[i] = x
            elif k == "wall_velocity":
                for f, vec in enumerate(v):
                    for a, x in enumerate(vec):
                        p.wall_velocity[f][a] = x
            elif k in ("tau", "smagorinsky_cs", "trt_magic"):
                setattr(p, k, v)
            else:
                raise LbmError(ERR_INVALID_ARG, f"unknown parameter {k}")
        self._c(load().lbm_set_params(self._h, C.byref(p)))

    def vdb_export(self, directory: str, frame: int, f32: bool = False) -> str:
        """Writes <directory>/velocity_<frame:06d>.vdb (lbm_vdb_export);
        returns the path."""
        rc = load().lbm_vdb_export(self._h, str(directory).encode(), frame, VDB_F32 if f32 else 0)
        if rc != OK:
            raise LbmError(rc, load().lbm_vdb_last_error().decode())
        return str(Path(directory) / f"velocity_{frame:06d}.vdb")

    def set_step_variant(self, nodes_per_thread: int) -> None:
        self._c(load().lbm_set_step_variant(self._h, nodes_per_thread))

    def read_mask(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint8)
        self._c(load().lbm_read_mask(self._h, _ptr(out), out.size))
        return out

    def set_iteration(self, iteration: int) -> None:
        self._c(load().lbm_set_iteration(self._h, iteration))

    def capture_save(self, root: str, frame: int, meta: dict | None = None,
                     full_state: bool = False) -> None:
        """F5: writes <root>/capture_<frame>/ (see lbm_capture_save)."""
        import json
        m = None if meta is None else json.dumps(meta).encode()
        self._c(load().lbm_capture_save(self._h, str(root).encode(), frame, m, int(full_state)))

    def capture_load(self, capture_dir: str, flags: int = 0) -> None:
        """F9: restores a capture (see lbm_capture_load)."""
        self._c(load().lbm_capture_load(self._h, str(capture_dir).encode(), flags))

    def set_closure(self, net: np.ndarray | None) -> None:
        """Installs a learned-closure network (float[CLOSURE_FLOATS]); None
        removes it."""
        if net is None:
            self._c(load().lbm_set_closure(self._h, None))
            return
        w = np.ascontiguousarray(net, dtype=np.float32).reshape(-1)
        if w.size != CLOSURE_FLOATS:
            raise LbmError(ERR_INVALID_ARG, f"network must have {CLOSURE_FLOATS} floats")
        self._c(load().lbm_set_closure(self._h, _ptr(w)))

    def set_closure_wait_limit(self, polls: int) -> None:
        """Testing hook: polls per tensor-core MMA wait (< 0: the default,
        0: give up at once); see lbm_set_closure_wait_limit."""
        self._c(load().lbm_set_closure_wait_limit(self._h, int(polls)))

    def read_classification(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        self._c(load().lbm_read_classification(self._h, _ptr(out), out.size))
        return out

    def init_equilibrium(self, rho0: float = 1.0, u0=(0.0, 0.0, 0.0)) -> None:
        u = (C.c_float * 3)(*u0)
        self._c(load().lbm_init_equilibrium(self._h, rho0, u))

    def init_from_moments(self, rho: np.ndarray, u: np.ndarray, fmt: int = U_F32X3) -> None:
        r = np.ascontiguousarray(rho, dtype=np.float32).reshape(-1)
        dt = np.uint16 if fmt == U_F16X4 else np.float32
        uu = np.ascontiguousarray(u, dtype=dt)
        self._c(load().lbm_init_from_moments(self._h, _ptr(r), _ptr(uu), fmt))

    def step(self, nsteps: int = 1) -> None:
        self._c(load().lbm_step(self._h, nsteps))

    def sync(self) -> None:
        self._c(load().lbm_sync(self._h))

    def read_moments(self, fmt: int = U_F32X3):
        rho = np.empty(self.n, np.float32)
        if fmt == U_F32X3:
            u = np.empty((self.n, 3), np.float32)
        elif fmt == U_F32X4:
            u = np.empty((self.n, 4), np.float32)
        else:
            u = np.empty((self.n, 4), np.uint16)
        self._c(load().lbm_read_moments(self._h, _ptr(rho), _ptr(u), fmt))
        return rho, u

    def device_moments(self):
        r, u = _P(), _P()
        self._c(load().lbm_device_moments(self._h, C.byref(r), C.byref(u)))
        return r.value, u.value

    def conservation(self) -> np.ndarray:
        out = (C.c_double * 4)()
        self._c(load().lbm_conservation(self._h, out))
        return np.array(out[:], np.float64)

    def conservation_async(self, out_ptr: int) -> None:
        """Queue the sums into out_ptr (four doubles in pinned host or
        device memory); valid once the stream reaches this point (sync)."""
        self._c(load().lbm_conservation_async(self._h, C.c_void_p(out_ptr)))

    def read_populations(self) -> np.ndarray:
        f = np.empty((19, self.n), np.float32)
        self._c(load().lbm_read_populations(self._h, _ptr(f), f.size))
        return f

    def write_populations(self, f: np.ndarray) -> None:
        ff = np.ascontiguousarray(f, dtype=np.float32)
        self._c(load().lbm_write_populations(self._h, _ptr(ff), ff.size))

    def info(self) -> Info:
        i = Info()
        i.struct_size = C.sizeof(Info)
        self._c(load().lbm_get_info(self._h, C.byref(i)))
        return i


class Batch:
    """Many independent physics-mode domains advanced together (lbm_batch)."""

    def __init__(self, descs):
        lib = load()
        self.descs = list(descs)
        arr = (Desc * len(self.descs))(*self.descs)
        h = _P()
        rc = lib.lbm_batch_create(arr, len(self.descs), C.byref(h))
        if rc != OK:
            raise LbmError(rc, lib.lbm_last_error(None).decode())
        self._h = h
        self.shapes = [(d.nx, d.ny, d.nz) for d in self.descs]

    def _c(self, rc: int) -> None:
        if rc != OK:
            raise LbmError(rc, load().lbm_batch_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n(self, d: int) -> int:
        nx, ny, nz = self.shapes[d]
        return nx * ny * nz

    def set_stream(self, stream_ptr) -> None:
        self._c(load().lbm_batch_set_stream(self._h, stream_ptr))

    def set_flags(self, d: int, mask: np.ndarray) -> None:
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        self._c(load().lbm_batch_set_flags(self._h, d, _ptr(m), m.size))

    def init_equilibrium(self, d: int = -1, rho0: float = 1.0, u0=(0.0, 0.0, 0.0)) -> None:
        self._c(load().lbm_batch_init_equilibrium(self._h, d, rho0, (C.c_float * 3)(*u0)))

    def init_from_moments(self, d: int, rho: np.ndarray, u: np.ndarray) -> None:
        r = np.ascontiguousarray(rho, dtype=np.float32).reshape(-1)
        uu = np.ascontiguousarray(u, dtype=np.float32)
        self._c(load().lbm_batch_init_from_moments(self._h, d, _ptr(r), _ptr(uu), U_F32X3))

    def step(self, nsteps: int = 1) -> None:
        self._c(load().lbm_batch_step(self._h, nsteps))

    def sync(self) -> None:
        self._c(load().lbm_batch_sync(self._h))

    def read_moments(self, d: int):
        n = self.n(d)
        rho = np.empty(n, np.float32)
        u = np.empty((n, 3), np.float32)
        self._c(load().lbm_batch_read_moments(self._h, d, _ptr(rho), _ptr(u), U_F32X3))
        return rho, u

    def read_populations(self, d: int) -> np.ndarray:
        f = np.empty((19, self.n(d)), np.float32)
        self._c(load().lbm_batch_read_populations(self._h, d, _ptr(f), f.size))
        return f

    def schedule(self) -> BatchSchedule:
        s = BatchSchedule()
        self._c(load().lbm_batch_get_schedule(self._h, C.byref(s)))
        return s

    def set_schedule(self, **kw) -> None:
        s = self.schedule()
        for k, v in kw.items():
            setattr(s, k, v)
        self._c(load().lbm_batch_set_schedule(self._h, C.byref(s)))

    def autotune(self, trial_steps: int = 10) -> BatchSchedule:
        s = BatchSchedule()
        s.struct_size = C.sizeof(BatchSchedule)
        self._c(load().lbm_batch_autotune(self._h, trial_steps, C.byref(s)))
        return s

    def info(self) -> BatchInfo:
        i = BatchInfo()
        i.struct_size = C.sizeof(BatchInfo)
        self._c(load().lbm_batch_get_info(self._h, C.byref(i)))
        return i


# --- mirror of the reference sim host ---------------------------------------

@dataclass(frozen=True)
class Tier:
    label: str
    nx: int
    ny: int
    nz: int


@dataclass(frozen=True)
class Preset:
    label: str
    naca: str
    angle_of_attack_deg: float
    u_inf: float
    tau: float


# TIERS and PRESETS of the reference (src/main.cpp:103-116, :122-135).
TIERS = (Tier("128^3 (Laptop)", 128, 128, 128),
         Tier("256x128x128 (Desktop)", 256, 128, 128),
         Tier("512x256x256 (Capture)", 512, 256, 256))
PRESETS = (Preset("NACA0012 - Low-Re", "0012", 4.0, 0.04, 0.60),
           Preset("NACA0012 - Med-Re", "0012", 8.0, 0.06, 0.55),
           Preset("NACA4412 - Med-Re", "4412", 6.0, 0.06, 0.55))
AIRFOIL_CHORD_CENTER_X_FRAC = 0.25
AIRFOIL_CHORD_LENGTH_FRAC = 0.25


def preset_u_inf(p: Preset):
    """update_u_inf_vector (src/main.cpp:1155-1160): |u| and AoA -> u_inf."""
    a = np.float32(p.angle_of_attack_deg) * np.float32(0.01745329251994329576923690768489)
    return (float(np.float32(p.u_inf) * np.float32(math.cos(a))),
            float(np.float32(p.u_inf) * np.float32(math.sin(a))), 0.0)


def preset_desc(preset_idx: int, nx: int, ny: int, nz: int) -> Desc:
    p = PRESETS[preset_idx]
    return default_desc(nx=nx, ny=ny, nz=nz, tau=p.tau, u_inf=preset_u_inf(p))


def apply_preset(lat: Lattice, preset_idx: int, device: bool = False) -> np.ndarray:
    """apply_preset (src/main.cpp:1167-1211): voxelise the airfoil, upload the
    mask, run the equilibrium init.  Returns the mask.  device=True makes the
    mask on the GPU (set_flags_naca; the same mask) and reads it back."""
    p = PRESETS[preset_idx]
    nx, ny, nz = lat.shape
    if device:
        lat.set_flags_naca(p.naca, AIRFOIL_CHORD_LENGTH_FRAC, AIRFOIL_CHORD_CENTER_X_FRAC,
                           p.angle_of_attack_deg)
        mask = lat.read_mask()
    else:
        mask = voxelize_naca(p.naca, nx, ny, nz, AIRFOIL_CHORD_LENGTH_FRAC, AIRFOIL_CHORD_CENTER_X_FRAC,
                             p.angle_of_attack_deg)
        lat.set_flags(mask)
    lat.init_equilibrium(1.0, tuple(lat.desc.u_inf))
    return mask


# ---- learned closure (include/lbm_closure.h) --------------------------------
# Device arguments are raw device pointers (ints), e.g. torch's data_ptr();
# `stream` is a cudaStream_t handle or None.

def round_bf16(a: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(a, dtype=np.float32)
    out = np.empty_like(x)
    _check(load().lbm_round_bf16(_ptr(x), _ptr(out), x.size))
    return out


def box_filter(d_rho: int, d_u: int, shape, factor: int, d_out: int, stream=None) -> None:
    nx, ny, nz = shape
    _check(load().lbm_box_filter(d_rho, d_u, nx, ny, nz, factor, d_out, stream))


def closure_samples(d_filt: int, shape, tau: float, cs0: float, seed: int, n_samples: int,
                    d_x: int, d_target: int, d_weight: int, stream=None) -> None:
    nx, ny, nz = shape
    _check(load().lbm_closure_samples(d_filt, nx, ny, nz, tau, cs0, seed, n_samples,
                                      d_x, d_target, d_weight, stream))


def closure_predict(net: np.ndarray, d_x: int, n: int, d_r: int, stream=None) -> None:
    w = np.ascontiguousarray(net, dtype=np.float32).reshape(-1)
    if w.size != CLOSURE_FLOATS:
        raise LbmError(ERR_INVALID_ARG, f"network must have {CLOSURE_FLOATS} floats")
    _check(load().lbm_closure_predict(_ptr(w), d_x, n, d_r, stream))


def adam_default(**kw) -> Adam:
    a = Adam()
    _check(load().lbm_adam_default(C.byref(a)))
    for k, v in kw.items():
        setattr(a, k, v)
    return a


class Trainer:
    """Fused forward/backward + Adam training of a closure network on the
    current CUDA device (lbm_trainer_*)."""

    def __init__(self, net: np.ndarray, adam: Adam | None = None):
        w = np.ascontiguousarray(net, dtype=np.float32).reshape(-1)
        if w.size != CLOSURE_FLOATS:
            raise LbmError(ERR_INVALID_ARG, f"network must have {CLOSURE_FLOATS} floats")
        self.adam = adam if adam is not None else adam_default()
        h = _P()
        _check(load().lbm_trainer_create(_ptr(w), C.byref(self.adam), C.byref(h)))
        self._h = h

    def _c(self, rc: int) -> None:
        if rc != OK:
            raise LbmError(rc, load().lbm_trainer_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().lbm_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream) -> None:
        self._c(load().lbm_trainer_set_stream(self._h, stream))

    def grad(self, d_x: int, d_target: int, d_weight: int, n: int, wscale: float):
        g = np.empty(CLOSURE_PARAMS, np.float32)
        loss = C.c_double()
        self._c(load().lbm_trainer_grad(self._h, d_x, d_target, d_weight, n, wscale, _ptr(g),
                                        C.byref(loss)))
        return g, loss.value

    def adam_step(self) -> None:
        self._c(load().lbm_trainer_adam_step(self._h))

    def fit(self, d_x: int, d_target: int, d_weight: int, n: int, batch: int, epochs: int,
            seed: int = 1) -> np.ndarray:
        losses = np.zeros(max(epochs, 1), np.float64)
        self._c(load().lbm_trainer_fit(self._h, d_x, d_target, d_weight, n, batch, epochs, seed,
                                       _ptr(losses)))
        return losses[:epochs]

    def net(self) -> np.ndarray:
        out = np.empty(CLOSURE_FLOATS, np.float32)
        self._c(load().lbm_trainer_get_net(self._h, _ptr(out)))
        return out


# ---- capture directories (include/lbm.h) -------------------------------------

def _cap_check(rc: int) -> None:
    if rc != OK:
        raise LbmError(rc, load().lbm_capture_last_error().decode())


def capture_write(root: str, frame: int, shape, rho: np.ndarray, vel_rgba16f: np.ndarray,
                  mask: np.ndarray, pops: np.ndarray | None = None, meta: dict | None = None) -> None:
    """Writes a capture from host arrays (no device needed)."""
    import json
    nx, ny, nz = shape
    n = nx * ny * nz
    r = np.ascontiguousarray(rho, np.float32).reshape(-1)
    v = np.ascontiguousarray(vel_rgba16f).view(np.uint16).reshape(-1)
    m = np.ascontiguousarray(mask, np.uint8).reshape(-1)
    if r.size != n or v.size != 4 * n or m.size != n:
        raise LbmError(ERR_INVALID_ARG, "capture_write: array sizes do not match the shape")
    p = None
    if pops is not None:
        p = np.ascontiguousarray(pops, np.float32).reshape(-1)
        if p.size != 19 * n:
            raise LbmError(ERR_INVALID_ARG, "capture_write: populations must be float[19][N]")
    mj = None if meta is None else json.dumps(meta).encode()
    _cap_check(load().lbm_capture_write(str(root).encode(), frame, mj, nx, ny, nz, _ptr(r), _ptr(v),
                                        _ptr(m), None if p is None else _ptr(p)))


def capture_read(capture_dir: str) -> dict:
    """Parses a capture: dict with the info fields and the arrays density
    float32[N], velocity uint16[N][4] (rgba16f bits), obstacle_mask
    uint8[N] and populations float32[19][N] (None if absent)."""
    info = CaptureInfo()
    info.struct_size = C.sizeof(CaptureInfo)
    d = str(capture_dir).encode()
    _cap_check(load().lbm_capture_read(d, C.byref(info), None, None, None, None))
    n = info.nx * info.ny * info.nz
    rho = np.empty(n, np.float32)
    vel = np.empty((n, 4), np.uint16)
    mask = np.empty(n, np.uint8)
    pops = np.empty((19, n), np.float32) if info.has_populations else None
    _cap_check(load().lbm_capture_read(d, C.byref(info), _ptr(rho), _ptr(vel), _ptr(mask),
                                       None if pops is None else _ptr(pops)))
    return {"shape": (info.nx, info.ny, info.nz), "frame": info.frame, "iteration": info.iteration,
            "mask_frame_invariant": bool(info.mask_frame_invariant), "density": rho, "velocity": vel,
            "obstacle_mask": mask, "populations": pops}


def capture_latest(root: str) -> str:
    buf = C.create_string_buffer(4096)
    _cap_check(load().lbm_capture_latest(str(root).encode(), buf, 4096))
    return buf.value.decode()


# ---- streamlines (include/lbm.h) -----------------------------------------------
STREAMLINE_COUNT = 10000
STREAMLINE_HISTORY = 64
STREAMLINE_RESEED_AGE = 256
STREAMLINE_SEED = 12345


def streamline_seed(count: int, history: int, shape, seed: int = STREAMLINE_SEED,
                    reseed_age: int = STREAMLINE_RESEED_AGE) -> np.ndarray:
    """Host seeding of the position ring: float32 [count][history][4]."""
    nx, ny, nz = shape
    out = np.empty((count, history, 4), np.float32)
    _check(load().lbm_streamline_seed(_ptr(out), count, history, nx, ny, nz, seed, reseed_age))
    return out


def streamline_advect(d_u: int, shape, d_positions: int, count: int, history: int, head: int,
                      frame: int, dt_render: float, reseed_age: int = STREAMLINE_RESEED_AGE,
                      round_f16: bool = True, stream=None) -> None:
    """One advect pass over device positions (float4 ring)."""
    nx, ny, nz = shape
    _check(load().lbm_streamline_advect(d_u, nx, ny, nz, d_positions, count, history, head, frame,
                                        dt_render, reseed_age, int(round_f16), stream))


# ---- velocity-magnitude raymarch (include/lbm.h) --------------------------------

def velmag_params(**kw) -> VelmagParams:
    p = VelmagParams()
    _check(load().lbm_velmag_params_default(C.byref(p)))
    for k, v in kw.items():
        if k in ("inv_view_proj", "camera_pos", "volume_min", "volume_max"):
            arr = getattr(p, k)
            vals = np.asarray(v, np.float32).reshape(-1)
            for i in range(len(arr)):
                arr[i] = float(vals[i])
        else:
            setattr(p, k, v)
    return p


def render_velmag(d_u: int, shape, params: VelmagParams, width: int, height: int, d_rgba: int,
                  stream=None) -> None:
    nx, ny, nz = shape
    _check(load().lbm_render_velmag(d_u, nx, ny, nz, C.byref(params), width, height, d_rgba, stream))


def colormap_lut() -> np.ndarray:
    out = np.empty((4, 256, 4), np.uint8)
    _check(load().lbm_colormap_lut(_ptr(out)))
    return out


def jitter_lut() -> np.ndarray:
    out = np.empty((256, 256), np.uint8)
    _check(load().lbm_jitter_lut(_ptr(out)))
    return out


def camera(eye, target, up=(0.0, 1.0, 0.0), fov_deg: float = 55.0, aspect: float = 16 / 9,
           near: float = 0.05, far: float = 4000.0) -> np.ndarray:
    """Inverse view-projection (column-major float[16]) of a right-handed
    look-at camera with a [0, 1]-depth perspective, the conventions of glm's
    lookAt and perspective under GLM_FORCE_DEPTH_ZERO_TO_ONE (the
    reference's defaults: fov 55 deg, near 0.05, far 4000,
    src/main.cpp:89-91)."""
    e, t, u = (np.asarray(a, np.float64) for a in (eye, target, up))
    f = (t - e) / np.linalg.norm(t - e)
    s = np.cross(f, u)
    s /= np.linalg.norm(s)
    uu = np.cross(s, f)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = s, uu, -f
    view[0, 3], view[1, 3], view[2, 3] = -s @ e, -uu @ e, f @ e
    th = np.tan(np.radians(fov_deg) / 2)
    proj = np.zeros((4, 4))
    proj[0, 0] = 1 / (aspect * th)
    proj[1, 1] = 1 / th
    proj[2, 2] = far / (near - far)
    proj[3, 2] = -1.0
    proj[2, 3] = -(far * near) / (far - near)
    inv = np.linalg.inv(proj @ view)
    return inv.T.reshape(-1).astype(np.float32)  # column-major


def write_ppm(path: str, rgba: np.ndarray) -> None:
    """Binary PPM of an RGBA float image [H][W][4] (colour over black,
    clamped to [0, 1])."""
    rgb = (np.clip(rgba[..., :3], 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
    h, w = rgb.shape[:2]
    with open(path, "wb") as f:
        f.write(f"P6 {w} {h} 255\n".encode())
        f.write(rgb.tobytes())
