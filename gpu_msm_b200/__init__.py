"""gpu_msm_b200 -- B200-native (sm_100a) BLS12-446 multi-scalar multiplication.

Python host mirror of the library's C-ABI (``include/gpu_msm_b200.h``).  The
compute path is the CUDA shared library ``libgpu_msm_b200.so`` built in-tree
by ``gpu_msm_b200/Makefile``; this module only loads it with ``ctypes`` and
moves buffers.  There is no CPU fallback: if the library is missing every
call raises.

Function names follow the reference's C-ABI and C++ API
(pdroalves/gpu_msm rust-api/include/rust_wrapper.h, include/curve.h):

* ``g1_msm_wrapper`` / ``g2_msm_wrapper`` -- host buffers, u64 scalars, same
  Montgomery conventions as the reference wrappers (G1 points in standard
  form, G2 points in Montgomery form);
* ``g1_msm`` / ``g2_msm`` -- host buffers, multi-limb scalars;
* ``msm_device`` -- device tensors, asynchronous on the current torch stream
  (the ``point_msm_async`` / ``point_msm_u64_async_g1`` analogue);
* ``projective_to_affine`` / ``affine_to_projective`` / ``from_montgomery`` ...
  the host-side point helpers of the reference's C wrapper.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpu_msm_b200.so")

# numpy dtypes byte-compatible with the C structs (include/gpu_msm_b200.h)
FP = np.dtype(("<u8", (7,)))
FP2 = np.dtype(("<u8", (2, 7)))
G1 = np.dtype([("x", "<u8", (7,)), ("y", "<u8", (7,)), ("infinity", "u1"), ("_pad", "u1", (7,))])
G2 = np.dtype([("x", "<u8", (2, 7)), ("y", "<u8", (2, 7)), ("infinity", "u1"), ("_pad", "u1", (7,))])
G1P = np.dtype([("X", "<u8", (7,)), ("Y", "<u8", (7,)), ("Z", "<u8", (7,))])
G2P = np.dtype([("X", "<u8", (2, 7)), ("Y", "<u8", (2, 7)), ("Z", "<u8", (2, 7))])

# u64 words per struct, for torch int64 views of device buffers
G1_WORDS, G2_WORDS, G1P_WORDS, G2P_WORDS = 15, 29, 21, 42

STATUS = {0: "ok", -1: "bad size or argument", -2: "stream creation failed", -3: "allocation failed",
          -4: "CUDA error", -5: "device consistency check failed"}

C_API = [
    # reference C-ABI (rust_wrapper.h)
    "affine_to_projective_g1_wrapper", "affine_to_projective_g2_wrapper",
    "projective_to_affine_g1_wrapper", "projective_to_affine_g2_wrapper",
    "g1_point_at_infinity_wrapper", "g2_point_at_infinity_wrapper",
    "g1_projective_point_at_infinity_wrapper", "g2_projective_point_at_infinity_wrapper",
    "g1_is_infinity_wrapper", "g2_is_infinity_wrapper", "g1_msm_wrapper", "g2_msm_wrapper",
    "g1_from_montgomery_wrapper", "g2_from_montgomery_wrapper", "fp_to_montgomery_wrapper",
    "init_device_generators",
    # additive entry points
    "g1_msm_limbs_wrapper", "g2_msm_limbs_wrapper", "gm_g1_msm_device", "gm_g2_msm_device",
    "gm_g1_msm_device_c", "gm_g2_msm_device_c", "gm_msm_default_window",
    "gm_fp_mont_mul_array", "gm_fp_mul_array", "gm_fp2_mont_mul_array", "gm_fp2_mul_array",
    "gm_fp_mont_sqr_array", "gm_fp_add_array", "gm_fp2_add_array",
    "gm_g1_msm_device_affine", "gm_g2_msm_device_affine",
    "gm_g1_to_montgomery_batch", "gm_g2_to_montgomery_batch",
    "gm_g1_generator_mul_batch", "gm_g2_generator_mul_batch", "gm_last_error",
    "gm_profile_enable", "gm_profile_collect", "gm_launch_count_reset", "gm_imad_probe",
    "gm_g1_sum_projective", "gm_g2_sum_projective", "gm_g1_msm_device_noalloc",
    "gm_bases_create", "gm_bases_destroy", "gm_bases_count", "gm_bases_precompute", "gm_msm_resident", "gm_batch_plan_create",
    "gm_batch_plan_run", "gm_batch_plan_destroy", "gm_batch_plan_bytes", "gm_batch_plan_classes",
    "gm_batch_plan_set_queue", "gm_batch_plan_create_tuned",
    "gm_batch_run", "gm_batch_workspace_bytes", "gm_g1_sum_projective_host", "gm_batch_run_ws",
    "gm_host_selftest", "gm_fp_elem", "gm_fp2_elem", "gm_g1_point_elem", "gm_g2_point_elem",
    "gm_g1_on_curve_batch", "gm_g2_on_curve_batch", "gm_g1_msm_host_async", "gm_g2_msm_host_async",
]


class MSMError(RuntimeError):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    """Load libgpu_msm_b200.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MSMError(f"CUDA library not built: {LIB_PATH} (run `make -C gpu_msm_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, u32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_int64
        for name in ("g1_msm_wrapper", "g2_msm_wrapper"):
            getattr(L, name).argtypes = [vp, vp, vp, i32, u32]
        for name in ("g1_msm_limbs_wrapper", "g2_msm_limbs_wrapper"):
            getattr(L, name).argtypes = [vp, vp, vp, i32, i32, u32, i32]
        for name in ("gm_g1_msm_device", "gm_g2_msm_device"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, vp, i32, i32]
        for name in ("gm_g1_msm_device_affine", "gm_g2_msm_device_affine"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, vp, i32, i32]
        for name in ("gm_g1_msm_device_c", "gm_g2_msm_device_c"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, vp, i32, i32, i32]
        L.gm_msm_default_window.argtypes = [i32, i64, i32]
        for name in ("gm_fp_mont_mul_array", "gm_fp_mul_array", "gm_fp2_mont_mul_array", "gm_fp2_mul_array",
                     "gm_fp_add_array", "gm_fp2_add_array"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, vp, i64]
        L.gm_fp_mont_sqr_array.argtypes = [vp, u32, vp, vp, i64]
        for name in ("gm_g1_to_montgomery_batch", "gm_g2_to_montgomery_batch"):
            getattr(L, name).argtypes = [vp, u32, vp, i32]
        for name in ("gm_g1_generator_mul_batch", "gm_g2_generator_mul_batch"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, i32, i32]
        L.gm_last_error.restype = ctypes.c_char_p
        for name in ("g1_is_infinity_wrapper", "g2_is_infinity_wrapper"):
            getattr(L, name).restype = ctypes.c_bool
        L.init_device_generators.argtypes = [vp, u32]
        L.gm_profile_enable.argtypes = [i32]
        L.gm_profile_collect.argtypes = [ctypes.c_char_p, i32, vp, i32]
        L.gm_launch_count_reset.restype = i64
        L.gm_imad_probe.argtypes = [vp, u32, i32, i32, vp, i64, vp]
        L.gm_g1_msm_device_noalloc.argtypes = [vp, u32, vp, vp, vp, i32, i32, vp]
        L.gm_bases_create.argtypes = [u32, i32, vp, i64, i32, vp]
        L.gm_bases_destroy.argtypes = [vp]
        L.gm_bases_precompute.argtypes = [vp, i32, i32]
        L.gm_bases_count.argtypes = [vp]
        L.gm_bases_count.restype = i64
        L.gm_msm_resident.argtypes = [vp, vp, i64, i32, vp, i32, vp, i32]
        L.gm_batch_plan_create.argtypes = [vp, i32, i32, vp, vp, vp, vp]
        L.gm_batch_plan_run.argtypes = [vp, vp, vp, vp]
        L.gm_batch_plan_destroy.argtypes = [vp]
        L.gm_batch_plan_bytes.argtypes = [vp]
        L.gm_batch_plan_bytes.restype = i64
        L.gm_batch_plan_classes.argtypes = [vp, vp, vp, i32]
        L.gm_batch_plan_set_queue.argtypes = [vp, i32]
        L.gm_batch_plan_create_tuned.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp]
        L.gm_batch_run.argtypes = [vp, vp, i32, i32, vp, vp, vp, vp, vp]
        L.gm_batch_run_ws.argtypes = [vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, i64]
        L.gm_g1_sum_projective_host.argtypes = [vp, vp, i32]
        L.gm_batch_workspace_bytes.argtypes = [vp, i32, i32, vp, vp]
        L.gm_batch_workspace_bytes.restype = i64
        for name in ("gm_g1_sum_projective", "gm_g2_sum_projective"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, i32]
        for name in ("gm_fp_elem", "gm_fp2_elem"):
            getattr(L, name).argtypes = [vp, u32, i32, vp, vp, vp, ctypes.c_uint64, vp]
        for name in ("gm_g1_point_elem", "gm_g2_point_elem"):
            getattr(L, name).argtypes = [vp, u32, i32, vp, vp, vp, vp, i32, ctypes.c_uint64]
        for name in ("gm_g1_on_curve_batch", "gm_g2_on_curve_batch"):
            getattr(L, name).argtypes = [vp, u32, vp, i64, vp]
        for name in ("gm_g1_msm_host_async", "gm_g2_msm_host_async"):
            getattr(L, name).argtypes = [vp, u32, vp, vp, vp, i32, i32, i32, vp]
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        msg = lib().gm_last_error().decode(errors="replace")
        raise MSMError(f"{what} failed: {rc} ({STATUS.get(rc, '?')}) {msg}")


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def _grp(group: int):
    if group == 1:
        return G1, G1P, "g1"
    if group == 2:
        return G2, G2P, "g2"
    raise ValueError("group must be 1 or 2")


def _scalars_2d(scalars, n: int) -> np.ndarray:
    s = np.ascontiguousarray(scalars, dtype=np.uint64)
    if s.ndim == 1:
        s = s.reshape(n, -1) if n else s.reshape(0, 1)
    if s.shape[0] != n:
        raise ValueError("scalars must have one row per point")
    return s


# ---------------------------------------------------------------------------
# host-buffer MSM
# ---------------------------------------------------------------------------

def g1_msm_wrapper(points: np.ndarray, scalars: np.ndarray, gpu_index: int = 0) -> np.ndarray:
    """Reference ``g1_msm_wrapper``: standard-form G1 points, u64 scalars."""
    pts = np.ascontiguousarray(points, dtype=G1)
    sc = np.ascontiguousarray(scalars, dtype=np.uint64).reshape(-1)
    out = np.zeros(1, dtype=G1P)
    _check(lib().g1_msm_wrapper(_p(out), _p(pts), _p(sc), len(pts), gpu_index), "g1_msm_wrapper")
    return out


def g2_msm_wrapper(points: np.ndarray, scalars: np.ndarray, gpu_index: int = 0) -> np.ndarray:
    """Reference ``g2_msm_wrapper``: Montgomery-form G2 points, u64 scalars."""
    pts = np.ascontiguousarray(points, dtype=G2)
    sc = np.ascontiguousarray(scalars, dtype=np.uint64).reshape(-1)
    out = np.zeros(1, dtype=G2P)
    _check(lib().g2_msm_wrapper(_p(out), _p(pts), _p(sc), len(pts), gpu_index), "g2_msm_wrapper")
    return out


def msm(points: np.ndarray, scalars: np.ndarray, group: int = 1, montgomery: bool = True,
        gpu_index: int = 0) -> np.ndarray:
    """sum_i scalars[i] * points[i] for host buffers; scalars are (n, limbs)
    little-endian u64.  Returns a projective point (Montgomery form)."""
    adt, pdt, g = _grp(group)
    pts = np.ascontiguousarray(points, dtype=adt)
    sc = _scalars_2d(scalars, len(pts))
    out = np.zeros(1, dtype=pdt)
    fn = getattr(lib(), f"{g}_msm_limbs_wrapper")
    _check(fn(_p(out), _p(pts), _p(sc), sc.shape[1], len(pts), gpu_index, 1 if montgomery else 0),
           f"{g}_msm_limbs_wrapper")
    return out


def msm_host_async(points: np.ndarray, scalars: np.ndarray, result: np.ndarray, group: int = 1,
                   montgomery: bool = True, gpu_index: int = 0, stream=None, err: np.ndarray = None):
    """Enqueue a host-buffer MSM on a torch CUDA stream (gm_g{1,2}_msm_host_async)
    and return at once.  points: structured G1/G2 array; scalars: uint64
    (n, limbs); result: a one-element G1P/G2P array receiving the projective
    sum; err: optional uint32 array of one element for the device check flag.
    Keep every buffer alive and read result only after the stream has passed
    the call.  Page-locked buffers (e.g. numpy views of pinned torch tensors)
    let the copies overlap other GPU work."""
    adt, pdt = (G1, G1P) if group == 1 else (G2, G2P)
    pts = np.asarray(points)
    if pts.dtype != adt or not pts.flags["C_CONTIGUOUS"]:
        raise ValueError("points: contiguous G1/G2 structured array")
    sc = np.asarray(scalars)
    if sc.dtype != np.uint64 or sc.ndim != 2 or sc.shape[0] != len(pts) or not sc.flags["C_CONTIGUOUS"]:
        raise ValueError("scalars: contiguous uint64 array (n, limbs)")
    if result.dtype != pdt or result.size != 1 or not result.flags["C_CONTIGUOUS"]:
        raise ValueError("result: one contiguous projective point")
    if err is not None and (err.dtype != np.uint32 or err.size != 1):
        raise ValueError("err: one uint32")
    fn = lib().gm_g1_msm_host_async if group == 1 else lib().gm_g2_msm_host_async
    _check(fn(_stream_handle(stream), gpu_index, _p(result), _p(pts), _p(sc), sc.shape[1], len(pts),
              1 if montgomery else 0, _p(err) if err is not None else None), "msm_host_async")


def g1_msm(points, scalars, montgomery=True, gpu_index=0):
    return msm(points, scalars, 1, montgomery, gpu_index)


def g2_msm(points, scalars, montgomery=True, gpu_index=0):
    return msm(points, scalars, 2, montgomery, gpu_index)


def default_window(group: int, n: int, scalar_limbs: int) -> int:
    return int(lib().gm_msm_default_window(group, n, scalar_limbs))


# ---------------------------------------------------------------------------
# host point helpers (reference c_wrapper.cu)
# ---------------------------------------------------------------------------

def projective_to_affine(proj: np.ndarray, group: int = 1) -> np.ndarray:
    adt, pdt, g = _grp(group)
    p = np.ascontiguousarray(proj, dtype=pdt).reshape(-1)
    out = np.zeros(len(p), dtype=adt)
    fn = getattr(lib(), f"projective_to_affine_{g}_wrapper")
    for i in range(len(p)):
        fn(ctypes.c_void_p(out.ctypes.data + i * adt.itemsize), ctypes.c_void_p(p.ctypes.data + i * pdt.itemsize))
    return out


def affine_to_projective(aff: np.ndarray, group: int = 1) -> np.ndarray:
    adt, pdt, g = _grp(group)
    a = np.ascontiguousarray(aff, dtype=adt).reshape(-1)
    out = np.zeros(len(a), dtype=pdt)
    fn = getattr(lib(), f"affine_to_projective_{g}_wrapper")
    for i in range(len(a)):
        fn(ctypes.c_void_p(out.ctypes.data + i * pdt.itemsize), ctypes.c_void_p(a.ctypes.data + i * adt.itemsize))
    return out


def from_montgomery(aff: np.ndarray, group: int = 1) -> np.ndarray:
    adt, _, g = _grp(group)
    a = np.ascontiguousarray(aff, dtype=adt).reshape(-1)
    out = np.zeros(len(a), dtype=adt)
    fn = getattr(lib(), f"{g}_from_montgomery_wrapper")
    for i in range(len(a)):
        fn(ctypes.c_void_p(out.ctypes.data + i * adt.itemsize), ctypes.c_void_p(a.ctypes.data + i * adt.itemsize))
    return out


def fp_to_montgomery(vals: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(vals, dtype=np.uint64).reshape(-1, 7)
    out = np.zeros_like(v)
    for i in range(len(v)):
        lib().fp_to_montgomery_wrapper(ctypes.c_void_p(out.ctypes.data + 56 * i), ctypes.c_void_p(v.ctypes.data + 56 * i))
    return out


def canonical_affine(proj: np.ndarray, group: int = 1) -> np.ndarray:
    """Projective (Montgomery) -> affine in standard form, the representation
    results are compared in."""
    return from_montgomery(projective_to_affine(proj, group), group)


# ---------------------------------------------------------------------------
# device-resident API (torch tensors as buffers, current torch stream)
# ---------------------------------------------------------------------------

def _require(t, cols, what, rows=None):
    """Shape/dtype/device checks before a device pointer crosses the ABI:
    a mismatched buffer would otherwise be read out of bounds on the GPU."""
    import torch
    if not isinstance(t, torch.Tensor) or t.dtype != torch.int64 or not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{what}: expected a contiguous int64 CUDA tensor")
    if t.dim() != 2 or (cols is not None and t.shape[1] != cols):
        raise ValueError(f"{what}: expected shape (n, {cols}), got {tuple(t.shape)}")
    if rows is not None and t.shape[0] != rows:
        raise ValueError(f"{what}: expected {rows} rows, got {t.shape[0]}")


def _stream_handle(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _dev_index(t) -> int:
    return t.device.index if t.device.index is not None else 0


def msm_device(points, scalars, group: int = 1, window_bits: int = 0, out=None, stream=None):
    """Asynchronous MSM on device tensors.

    points:  int64 tensor (n, 15) [G1Point] or (n, 29) [G2Point], Montgomery form
    scalars: int64 tensor (n, limbs), little-endian u64 limbs
    returns: int64 tensor (21,) or (42,) -- projective result, Montgomery form
    """
    import torch
    _require(points, G1_WORDS if group == 1 else G2_WORDS, "points")
    n = points.shape[0]
    _require(scalars, None, "scalars", rows=n)
    limbs = scalars.shape[1]
    if not 1 <= limbs <= 8:
        raise ValueError("scalars: 1..8 limbs per scalar")
    if scalars.device != points.device:
        raise ValueError("points and scalars must be on the same device")
    words = G1P_WORDS if group == 1 else G2P_WORDS
    if out is None:
        out = torch.empty(words, dtype=torch.int64, device=points.device)
    if out.numel() < words or out.dtype != torch.int64 or out.device != points.device:
        raise ValueError("out: int64 tensor of the result size on the points' device")
    fn = lib().gm_g1_msm_device_c if group == 1 else lib().gm_g2_msm_device_c
    _check(fn(_stream_handle(stream), _dev_index(points), ctypes.c_void_p(out.data_ptr()),
              ctypes.c_void_p(points.data_ptr()), ctypes.c_void_p(scalars.data_ptr()), limbs, n, window_bits),
           "msm_device")
    return out


def msm_device_affine(points, scalars, group: int = 1, out=None, stream=None):
    """MSM with an affine result (reference layout, Montgomery form, infinity
    flag), the device form of point_msm_async<G1Point>/<G2Point>.  Returns an
    int64 tensor of G1_WORDS / G2_WORDS words."""
    import torch
    _require(points, G1_WORDS if group == 1 else G2_WORDS, "points")
    n = points.shape[0]
    _require(scalars, None, "scalars", rows=n)
    limbs = scalars.shape[1]
    words = G1_WORDS if group == 1 else G2_WORDS
    if out is None:
        out = torch.empty(words, dtype=torch.int64, device=points.device)
    fn = lib().gm_g1_msm_device_affine if group == 1 else lib().gm_g2_msm_device_affine
    _check(fn(_stream_handle(stream), _dev_index(points), ctypes.c_void_p(out.data_ptr()),
              ctypes.c_void_p(points.data_ptr()), ctypes.c_void_p(scalars.data_ptr()), limbs, n), "msm_device_affine")
    return out


NOALLOC_MAX_POINTS = 4096


def msm_device_noalloc(points, scalars, out=None, err=None, stream=None):
    """G1 MSM through gm_g1_msm_device_noalloc, for callers that cannot
    allocate device memory per call: the workspace is fixed in the library's
    device image, so at most 4096 points per call.  Calls that overlap on the
    GPU share that workspace and race; keep them on one stream.  err: optional
    int32 CUDA tensor of one element that receives the consistency flag
    (0 = ok) on the stream."""
    import torch
    _require(points, G1_WORDS, "points")
    n = points.shape[0]
    _require(scalars, None, "scalars", rows=n)
    if out is None:
        out = torch.empty(G1P_WORDS, dtype=torch.int64, device=points.device)
    if out.numel() < G1P_WORDS or out.dtype != torch.int64 or out.device != points.device:
        raise ValueError("out: int64 tensor of the result size on the points' device")
    if err is not None and (err.dtype != torch.int32 or err.numel() < 1 or err.device != points.device):
        raise ValueError("err: int32 tensor of one element on the points' device")
    _check(lib().gm_g1_msm_device_noalloc(_stream_handle(stream), _dev_index(points), ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(points.data_ptr()), ctypes.c_void_p(scalars.data_ptr()),
                                          scalars.shape[1], n, _ptr_or_null(err)), "msm_device_noalloc")
    return out


def sum_projective(points, group: int = 1, out=None, stream=None):
    """Device sum of projective points (int64 tensor (k, 21) or (k, 42))."""
    import torch
    words = G1P_WORDS if group == 1 else G2P_WORDS
    _require(points, words, "points")
    if out is None:
        out = torch.empty(words, dtype=torch.int64, device=points.device)
    if out.numel() < words or out.dtype != torch.int64:
        raise ValueError("out: int64 tensor of the result size")
    fn = lib().gm_g1_sum_projective if group == 1 else lib().gm_g2_sum_projective
    _check(fn(_stream_handle(stream), _dev_index(points), ctypes.c_void_p(out.data_ptr()),
              ctypes.c_void_p(points.data_ptr()), points.shape[0]), "sum_projective")
    return out


def sum_projective_host(points: np.ndarray) -> np.ndarray:
    """Host-side sum of G1 projective points (numpy G1P array)."""
    pts = np.ascontiguousarray(points, dtype=G1P).reshape(-1)
    out = np.zeros(1, dtype=G1P)
    _check(lib().gm_g1_sum_projective_host(_p(out), _p(pts), len(pts)), "gm_g1_sum_projective_host")
    return out


def generator_mul_batch(scalars, group: int = 1, stream=None):
    """out[i] = scalars[i] * G (canonical Montgomery affine) on the device."""
    import torch
    _require(scalars, None, "scalars")
    n = scalars.shape[0]
    limbs = scalars.shape[1]
    if not 1 <= limbs <= 8:
        raise ValueError("scalars: 1..8 limbs per scalar")
    words = G1_WORDS if group == 1 else G2_WORDS
    out = torch.empty((n, words), dtype=torch.int64, device=scalars.device)
    fn = lib().gm_g1_generator_mul_batch if group == 1 else lib().gm_g2_generator_mul_batch
    _check(fn(_stream_handle(stream), _dev_index(scalars), ctypes.c_void_p(out.data_ptr()),
              ctypes.c_void_p(scalars.data_ptr()), limbs, n), "generator_mul_batch")
    return out


def to_montgomery_batch(points, group: int = 1, stream=None):
    _require(points, G1_WORDS if group == 1 else G2_WORDS, "points")
    fn = lib().gm_g1_to_montgomery_batch if group == 1 else lib().gm_g2_to_montgomery_batch
    _check(fn(_stream_handle(stream), _dev_index(points), ctypes.c_void_p(points.data_ptr()), points.shape[0]),
           "to_montgomery_batch")
    return points


def field_mul_array(a, b, op: str = "fp_mont_mul", out=None, stream=None):
    """Element-wise field products on device tensors of shape (n, 7) [Fp] or
    (n, 14) [Fp2], int64.  op: fp_mont_mul | fp_mul | fp_add | fp2_mont_mul | fp2_mul |
    fp2_add."""
    import torch
    cols = 7 if op.startswith("fp_") else 14
    _require(a, cols, "a")
    _require(b, cols, "b", rows=a.shape[0])
    if out is None:
        out = torch.empty_like(a)
    _require(out, cols, "out", rows=a.shape[0])
    fn = getattr(lib(), f"gm_{op}_array")
    _check(fn(_stream_handle(stream), _dev_index(a), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(a.data_ptr()),
              ctypes.c_void_p(b.data_ptr()), a.shape[0]), op)
    return out


def field_sqr_array(a, out=None, stream=None):
    """Element-wise Montgomery squares a^2 R^-1 of an (n, 7) int64 device
    tensor of Fp elements (the dedicated squaring of the point formulas)."""
    import torch
    _require(a, 7, "a")
    if out is None:
        out = torch.empty_like(a)
    _require(out, 7, "out", rows=a.shape[0])
    _check(lib().gm_fp_mont_sqr_array(_stream_handle(stream), _dev_index(a), ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(a.data_ptr()), a.shape[0]), "fp_mont_sqr")
    return out


# Single-element operations (gm_fp_elem, gm_fp2_elem, gm_g{1,2}_point_elem):
# op names in the order of GM_FP_*, GM_FP2_* and GM_PT_* of
# include/gpu_msm_b200.h.  They back the reference's stream APIs
# fp_*_async / fp2_*_async / point_*_async (include/fp.h:158-204,
# include/fp2.h:99-133, include/curve.h:156-211).
FP_OPS = ("add", "sub", "mul", "neg", "inv", "div", "copy", "zero", "one", "to_mont", "from_mont", "mont_mul",
          "cmp", "is_zero", "is_one", "cmov", "sqrt", "is_qr", "pow_u64")
FP2_OPS = ("add", "sub", "mul", "square", "neg", "conjugate", "inv", "div", "copy", "mul_by_i", "frobenius",
           "cmp", "is_zero", "is_one", "cmov", "mont_mul")
POINT_OPS = ("add", "double", "neg", "scalar_mul", "scalar_mul_u64", "to_mont", "from_mont", "at_infinity")


def _ptr_or_null(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def field_elem(op: str, a=None, b=None, c=None, arg: int = 0, fp2: bool = False, flag=None, stream=None):
    """One Fp (or Fp2) element operation on int64 device tensors of shape
    (1, 7) [(1, 14) for Fp2], asynchronous on the current torch stream.
    ``c`` receives the result (allocated when None; read too by cmov);
    ``flag`` (an int32 device tensor of one element, allocated when None)
    receives cmp / is_zero / is_one / is_qr / sqrt's answer.  mul, inv, div,
    square, sqrt, is_qr and pow_u64 work on standard-form values.
    Returns (c, flag)."""
    import torch
    ops = FP2_OPS if fp2 else FP_OPS
    code = ops.index(op)
    cols = 14 if fp2 else 7
    ref = a if a is not None else c
    for t, what in ((a, "a"), (b, "b"), (c, "c")):
        if t is not None:
            _require(t, cols, what, rows=1)
    dev = ref.device if ref is not None else torch.device("cuda", torch.cuda.current_device())
    if c is None:
        c = torch.zeros((1, cols), dtype=torch.int64, device=dev)
    if flag is None:
        flag = torch.zeros(1, dtype=torch.int32, device=dev)
    fn = lib().gm_fp2_elem if fp2 else lib().gm_fp_elem
    _check(fn(_stream_handle(stream), _dev_index(c), code, _ptr_or_null(c), _ptr_or_null(a), _ptr_or_null(b),
              ctypes.c_uint64(arg & 0xFFFFFFFFFFFFFFFF), ctypes.c_void_p(flag.data_ptr())),
           ("fp2_" if fp2 else "fp_") + op)
    return c, flag


def point_elem(op: str, p=None, q=None, scalar=None, scalar_u64: int = 0, group: int = 1, out=None, stream=None):
    """One affine point operation (gm_g{1,2}_point_elem) on int64 device
    tensors of shape (1, 15) [G1Point] or (1, 29) [G2Point], Montgomery form;
    ``scalar`` is an int64 device tensor (1, limbs) for scalar_mul.  Returns
    the result tensor."""
    import torch
    code = POINT_OPS.index(op)
    cols = G1_WORDS if group == 1 else G2_WORDS
    for t, what in ((p, "p"), (q, "q")):
        if t is not None:
            _require(t, cols, what, rows=1)
    limbs = 0
    if scalar is not None:
        _require(scalar, None, "scalar", rows=1)
        limbs = scalar.shape[1]
    ref = p if p is not None else out
    dev = ref.device if ref is not None else torch.device("cuda", torch.cuda.current_device())
    if out is None:
        out = torch.zeros((1, cols), dtype=torch.int64, device=dev)
    _require(out, cols, "out", rows=1)
    fn = lib().gm_g1_point_elem if group == 1 else lib().gm_g2_point_elem
    _check(fn(_stream_handle(stream), _dev_index(out), code, ctypes.c_void_p(out.data_ptr()), _ptr_or_null(p),
              _ptr_or_null(q), _ptr_or_null(scalar), limbs, ctypes.c_uint64(scalar_u64 & 0xFFFFFFFFFFFFFFFF)),
           f"g{group}_point_{op}")
    return out


def on_curve(points, group: int = 1, stream=None):
    """uint8 device tensor (n,): 1 where the affine point (int64 device tensor
    (n, 15) [G1Point] or (n, 29) [G2Point], Montgomery form) satisfies
    y^2 = x^3 + 1 (G1) / x^3 + (1 + i) (G2) or is at infinity."""
    import torch
    _require(points, G1_WORDS if group == 1 else G2_WORDS, "points")
    ok = torch.empty(points.shape[0], dtype=torch.uint8, device=points.device)
    fn = lib().gm_g1_on_curve_batch if group == 1 else lib().gm_g2_on_curve_batch
    _check(fn(_stream_handle(stream), _dev_index(points), ctypes.c_void_p(points.data_ptr()), points.shape[0],
              ctypes.c_void_p(ok.data_ptr())), "on_curve")
    return ok


def to_numpy_points(t, group: int = 1) -> np.ndarray:
    """Copy an int64 device/host tensor of points to a numpy structured array."""
    arr = t.detach().cpu().numpy().view(np.uint64)
    adt = G1 if group == 1 else G2
    return np.ascontiguousarray(arr).view(adt).reshape(-1)


def to_numpy_proj(t, group: int = 1) -> np.ndarray:
    arr = t.detach().cpu().numpy().view(np.uint64)
    pdt = G1P if group == 1 else G2P
    return np.ascontiguousarray(arr).view(pdt).reshape(-1)


# ---------------------------------------------------------------------------
# measurement hooks
# ---------------------------------------------------------------------------

def profile_enable(on: bool = True):
    lib().gm_profile_enable(1 if on else 0)


def profile_collect(max_phases: int = 4096):
    """[(phase, ms), ...] for the MSMs run since profiling was enabled
    (synchronises the recorded events)."""
    names = ctypes.create_string_buffer(64 * max_phases)
    ms = np.zeros(max_phases, dtype=np.float32)
    n = lib().gm_profile_collect(names, len(names), ctypes.c_void_p(ms.ctypes.data), max_phases)
    labels = names.value.decode().split(",") if n else []
    return list(zip(labels, ms[:n].tolist()))


def launch_count_reset() -> int:
    return int(lib().gm_launch_count_reset())


def imad_probe(iters: int, sink, stream=None, mode: int = 0) -> int:
    """Launch the multiply-add throughput probe (mode 0: mad.lo/mad.hi mix,
    1: mad.lo only); returns instructions per launch."""
    import torch
    if not (isinstance(sink, torch.Tensor) and sink.is_cuda and sink.dtype == torch.int32):
        raise ValueError("sink: int32 CUDA tensor")
    cnt = ctypes.c_int64(0)
    _check(lib().gm_imad_probe(_stream_handle(stream), _dev_index(sink), iters, mode, ctypes.c_void_p(sink.data_ptr()),
                               sink.numel(), ctypes.byref(cnt)), "imad_probe")
    return cnt.value


# ---------------------------------------------------------------------------
# resident base tables and batched MSMs
# ---------------------------------------------------------------------------

class ResidentBases:
    """A base table packed once on the device (``gm_bases_create``).

    points: int64 CUDA tensor (n, 15) [G1Point] or (n, 29) [G2Point] in the
    reference layout; Montgomery form unless montgomery=False."""

    def __init__(self, points, group: int = 1, montgomery: bool = True):
        _require(points, G1_WORDS if group == 1 else G2_WORDS, "points")
        self.group = group
        self.n = points.shape[0]
        self.device = points.device
        h = ctypes.c_void_p()
        _check(lib().gm_bases_create(_dev_index(points), group, ctypes.c_void_p(points.data_ptr()), self.n,
                                     1 if montgomery else 0, ctypes.byref(h)), "gm_bases_create")
        self.handle = h
        self.precomputed = []   # window widths with a fixed-base table

    def precompute(self, window_bits: int, scalar_limbs: int = 5):
        """Build the fixed-base window table for window width window_bits
        (``gm_bases_precompute``): 2^(c w) * P_i for every window, so MSMs of
        that width need one bucket set and no window doublings.  Blocks."""
        _check(lib().gm_bases_precompute(self.handle, int(window_bits), int(scalar_limbs)), "gm_bases_precompute")
        if window_bits not in self.precomputed:
            self.precomputed.append(int(window_bits))
        return self

    def windows_for(self, sizes, scalar_limbs: int = 5):
        """Per-MSM window widths to pass to a plan: 0 (the library picks the
        cheapest fixed-base table) when the set has tables, else the tuned
        widths."""
        if self.precomputed:
            return [0] * len(sizes)
        return [tuned_window(self.group, int(s), scalar_limbs) for s in sizes]

    def msm(self, scalars, offset: int = 0, n: int = None, window_bits: int = 0, out=None, stream=None):
        """Asynchronous MSM over entries [offset, offset + n)."""
        import torch
        n = scalars.shape[0] if n is None else n
        _require(scalars, None, "scalars", rows=n)
        if offset < 0 or offset + n > self.n:
            raise ValueError("range outside the base table")
        words = G1P_WORDS if self.group == 1 else G2P_WORDS
        if out is None:
            out = torch.empty(words, dtype=torch.int64, device=self.device)
        _check(lib().gm_msm_resident(_stream_handle(stream), self.handle, offset, n, ctypes.c_void_p(scalars.data_ptr()),
                                     scalars.shape[1], ctypes.c_void_p(out.data_ptr()), window_bits),
               "gm_msm_resident")
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().gm_bases_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_WINDOW_TABLE = None


def window_table() -> dict:
    """The autotuner's table (gpu_msm_b200/window_table.json), or {}."""
    global _WINDOW_TABLE
    if _WINDOW_TABLE is None:
        import json
        path = os.path.join(_HERE, "window_table.json")
        try:
            with open(path) as f:
                _WINDOW_TABLE = json.load(f)
        except (OSError, ValueError):
            _WINDOW_TABLE = {}
    return _WINDOW_TABLE


def tuned_params(group: int, n: int, scalar_limbs: int = 5):
    """(window width, accumulation slice waves, sort points per thread) for an
    MSM of n points: the autotuned values of its size class floor(log2 n)
    when tuned, else (cost model, 1, 4).  Table entries are either a width
    or {"c": .., "slice_waves": .., "sort_ppt": ..}."""
    tab = window_table().get(f"g{group}", {})
    e = max(0, int(n).bit_length() - 1)
    v = tab.get(str(e))
    if isinstance(v, dict):
        return int(v["c"]), int(v.get("slice_waves", 1)), int(v.get("sort_ppt", 4))
    if v is not None:
        return int(v), 1, 4
    return default_window(group, n, scalar_limbs), 1, 4


def tuned_window(group: int, n: int, scalar_limbs: int = 5) -> int:
    """Window width for an MSM of n points: the autotuned value for its size
    class floor(log2 n) when tuned, else the library's cost model."""
    return tuned_params(group, n, scalar_limbs)[0]


class BatchPlan:
    """A fixed batch of MSMs over a resident table (``gm_batch_plan_*``).

    sizes[i] points for MSM i starting at table entry base_offsets[i];
    window_bits[i] (0: cost model).  ``run`` enqueues the whole batch on the
    current (or given) stream; it only launches kernels, so it can be captured
    in a CUDA graph and replayed with new scalars in the same tensor."""

    def __init__(self, bases: ResidentBases, sizes, base_offsets=None, window_bits=None, scalar_limbs: int = 5,
                 tuning=None):
        """tuning: None = the autotuned (slice waves, sort points per thread)
        of each MSM's size class; or an int32 array (count, 2)."""
        self.bases = bases
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int64)
        self.count = len(self.sizes)
        self.total = int(self.sizes.sum())
        self.limbs = scalar_limbs
        offs = None if base_offsets is None else np.ascontiguousarray(base_offsets, dtype=np.int64)
        if window_bits is None:
            window_bits = bases.windows_for(self.sizes, scalar_limbs)
        wins = np.ascontiguousarray(window_bits, dtype=np.int32)
        if tuning is None:
            tuning = [tuned_params(bases.group, int(n), scalar_limbs)[1:] for n in self.sizes]
        tun = np.ascontiguousarray(np.asarray(tuning, dtype=np.int32).reshape(self.count, 2))
        h = ctypes.c_void_p()
        _check(lib().gm_batch_plan_create_tuned(bases.handle, scalar_limbs, self.count, _p(self.sizes),
                                                None if offs is None else _p(offs), _p(wins), _p(tun),
                                                ctypes.byref(h)), "gm_batch_plan_create_tuned")
        self.handle = h
        self._keep = (offs, wins, tun)

    @property
    def workspace_bytes(self) -> int:
        return int(lib().gm_batch_plan_bytes(self.handle))

    def set_queue(self, on: bool = True):
        """Accumulation mode (gm_batch_plan_set_queue): True (the default) =
        every class's accumulation in one persistent launch over a device work
        queue; False = one pipeline per window class on its own stream.  Same
        results."""
        _check(lib().gm_batch_plan_set_queue(self.handle, 1 if on else 0), "gm_batch_plan_set_queue")
        return self

    def classes(self):
        w = np.zeros(64, dtype=np.int32)
        c = np.zeros(64, dtype=np.int32)
        k = lib().gm_batch_plan_classes(self.handle, _p(w), _p(c), 64)
        return list(zip(w[:k].tolist(), c[:k].tolist()))

    def run(self, scalars, out=None, stream=None):
        import torch
        _require(scalars, self.limbs, "scalars", rows=self.total)
        words = G1P_WORDS if self.bases.group == 1 else G2P_WORDS
        if out is None:
            out = torch.empty((self.count, words), dtype=torch.int64, device=scalars.device)
        _check(lib().gm_batch_plan_run(self.handle, _stream_handle(stream), ctypes.c_void_p(scalars.data_ptr()),
                                       ctypes.c_void_p(out.data_ptr())), "gm_batch_plan_run")
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().gm_batch_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_run(bases: ResidentBases, sizes, scalars, base_offsets=None, window_bits=None, out=None, stream=None,
              workspace=None):
    """One batch without a plan (``gm_batch_run``): classes in order on the
    stream, for batches whose shape changes on every call.  workspace: None
    takes the device memory from the library's stream-ordered pool for this
    run; or a uint8 device tensor of at least ``batch_workspace_bytes`` bytes
    (``gm_batch_run_ws``), in use until the stream has run the batch."""
    import torch
    sizes = np.ascontiguousarray(sizes, dtype=np.int64)
    total = int(sizes.sum())
    _require(scalars, None, "scalars", rows=total)
    if window_bits is None:
        window_bits = bases.windows_for(sizes, scalars.shape[1])
    wins = np.ascontiguousarray(window_bits, dtype=np.int32)
    offs = None if base_offsets is None else np.ascontiguousarray(base_offsets, dtype=np.int64)
    words = G1P_WORDS if bases.group == 1 else G2P_WORDS
    if out is None:
        out = torch.empty((len(sizes), words), dtype=torch.int64, device=scalars.device)
    args = (_stream_handle(stream), bases.handle, scalars.shape[1], len(sizes), _p(sizes),
            None if offs is None else _p(offs), _p(wins), ctypes.c_void_p(scalars.data_ptr()),
            ctypes.c_void_p(out.data_ptr()))
    if workspace is None:
        _check(lib().gm_batch_run(*args), "gm_batch_run")
    else:
        if workspace.dtype != torch.uint8 or workspace.device != scalars.device:
            raise ValueError("workspace: uint8 tensor on the scalars' device")
        _check(lib().gm_batch_run_ws(*args, ctypes.c_void_p(workspace.data_ptr()), workspace.numel()),
               "gm_batch_run_ws")
    return out


def batch_workspace_bytes(bases: ResidentBases, sizes, window_bits=None, scalar_limbs: int = 5) -> int:
    sizes = np.ascontiguousarray(sizes, dtype=np.int64)
    if window_bits is None:
        window_bits = bases.windows_for(sizes, scalar_limbs)
    wins = np.ascontiguousarray(window_bits, dtype=np.int32)
    v = int(lib().gm_batch_workspace_bytes(bases.handle, scalar_limbs, len(sizes), _p(sizes), _p(wins)))
    if v < 0:
        raise MSMError("gm_batch_workspace_bytes: bad batch")
    return v
