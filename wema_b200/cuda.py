"""ctypes binding of libwema_cuda (the product library) for tests and the
benchmark.  Device buffers are torch CUDA tensors (torch is plumbing only:
allocation and streams); every computation runs in the library's kernels.

There is no fallback: if the library or a GPU is missing, using it raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _build

READ_GRAY_IN, READ_GRAY_OUT, READ_ORIG6, READ_DELTA6, READ_AMP6, READ_LOWPASS, \
    READ_THRESHOLD, READ_MAGSUM = range(8)
THR_SINGLE, THR_BATCH = 0, 1


class Config(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("fps", C.c_float),
                ("amp_factor", C.c_float), ("f_low", C.c_float), ("f_high", C.c_float),
                ("temporal_window", C.c_int), ("edge_aware", C.c_int),
                ("bilateral_temp", C.c_int), ("color_mode", C.c_int), ("use_iir", C.c_int),
                ("threshold_form", C.c_int), ("device", C.c_int), ("iir_state_fp64", C.c_int),
                ("ring_fp16", C.c_int), ("planes_fp16", C.c_int)]


_lib = None


class SessionStatus(C.Structure):
    """wema_cuda_session_status"""
    _fields_ = [("state", C.c_int), ("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("dropped", C.c_longlong), ("state_bytes", C.c_size_t),
                ("admission_wait_ms", C.c_double)]


class ServeStats(C.Structure):
    """wema_cuda_serve_stats"""
    _fields_ = [("seconds", C.c_double), ("ticks", C.c_longlong), ("frames", C.c_longlong),
                ("launches", C.c_longlong), ("mpix_frames", C.c_double),
                ("latency_p50_ms", C.c_float), ("latency_p99_ms", C.c_float),
                ("latency_max_ms", C.c_float), ("admission_wait_p50_ms", C.c_float),
                ("admission_wait_max_ms", C.c_float), ("sessions_admitted", C.c_longlong),
                ("sessions_live", C.c_int), ("sessions_queued", C.c_int),
                ("bytes_used", C.c_size_t), ("budget_bytes", C.c_size_t),
                ("tick_host_ms_mean", C.c_float), ("tick_host_ms_max", C.c_float),
                ("tick_span_ms_mean", C.c_float), ("tick_span_ms_max", C.c_float),
                ("admit_ms_max", C.c_float), ("retire_ms_max", C.c_float)]


SESSION_QUEUED, SESSION_LIVE, SESSION_CLOSED, SESSION_FAILED = 0, 1, 2, 3


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.cuda_lib_path()
        if not os.path.exists(path):
            raise RuntimeError(f"libwema_cuda not built ({path}); run __graft_entry__.build()")
        L = C.CDLL(path)
        vp, i, f, sz = C.c_void_p, C.c_int, C.c_float, C.c_size_t
        L.wema_cuda_last_error.restype = C.c_char_p
        L.wema_cuda_config_default.argtypes = [C.POINTER(Config), i, i, f]
        L.wema_cuda_session_bytes.argtypes = [C.POINTER(Config)]
        L.wema_cuda_session_bytes.restype = sz
        L.wema_cuda_session_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
        L.wema_cuda_session_destroy.argtypes = [vp]
        L.wema_cuda_process_u8.argtypes = [vp, vp, vp, vp]
        L.wema_cuda_process_u8_async.argtypes = [vp, vp, vp, vp, vp]
        L.wema_cuda_set_inspect.argtypes = [vp, i]
        L.wema_cuda_process_f32.argtypes = [vp, vp, vp, vp, vp]
        L.wema_cuda_process_host_u8.argtypes = [vp, vp, vp]
        L.wema_cuda_session_sync.argtypes = [vp]
        L.wema_cuda_session_frames_processed.argtypes = [vp]
        L.wema_cuda_session_read.argtypes = [vp, i, i, vp, sz]
        L.wema_cuda_session_read.restype = C.c_long
        L.wema_cuda_threshold_flat.argtypes = [vp, sz, i, vp, vp, vp]
        L.wema_cuda_threshold_flat_noalloc.argtypes = [vp, sz, i, vp, vp, vp]
        L.wema_cuda_set_timing.argtypes = [vp, i]
        L.wema_cuda_stage_times.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        L.wema_cuda_session_launches.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.wema_cuda_batch_stream_bytes.argtypes = [C.POINTER(Config)]
        L.wema_cuda_batch_stream_bytes.restype = sz
        L.wema_cuda_batch_create.argtypes = [i, i, C.POINTER(vp)]
        L.wema_cuda_batch_destroy.argtypes = [vp]
        L.wema_cuda_batch_destroy.restype = None
        L.wema_cuda_batch_add.argtypes = [vp, C.POINTER(Config), C.POINTER(i)]
        L.wema_cuda_batch_remove.argtypes = [vp, i]
        L.wema_cuda_batch_tick.argtypes = [vp, C.POINTER(i), C.POINTER(vp), C.POINTER(vp), i, vp, vp]
        L.wema_cuda_batch_sync.argtypes = [vp]
        L.wema_cuda_autotune.argtypes = [i, C.c_char_p, sz]
        L.wema_cuda_set_iir_positions.argtypes = [i, i]
        L.wema_cuda_get_iir_positions.argtypes = [i]
        L.wema_cuda_set_guided_rows.argtypes = [i, i]
        L.wema_cuda_get_guided_rows.argtypes = [i]
        L.wema_cuda_set_dwt_variant.argtypes = [i, i, i]
        L.wema_cuda_get_dwt_variant.argtypes = [i, i]
        L.wema_cuda_batch_tick_host.argtypes = [vp, C.POINTER(i), C.POINTER(vp), C.POINTER(vp), i, vp, vp]
        L.wema_cuda_session_snapshot_bytes.argtypes = [vp]
        L.wema_cuda_session_snapshot_bytes.restype = sz
        L.wema_cuda_session_snapshot.argtypes = [vp, vp, sz]
        L.wema_cuda_session_restore.argtypes = [vp, vp, sz]
        L.wema_cuda_batch_snapshot_bytes.argtypes = [vp, i]
        L.wema_cuda_batch_snapshot_bytes.restype = sz
        L.wema_cuda_batch_snapshot.argtypes = [vp, i, vp, sz]
        L.wema_cuda_batch_restore.argtypes = [vp, i, vp, sz]
        L.wema_cuda_batch_set_timing.argtypes = [vp, i]
        L.wema_cuda_batch_set_host_overlap.argtypes = [vp, i]
        L.wema_cuda_batch_set_graphs.argtypes = [vp, i]
        L.wema_cuda_batch_set_groups.argtypes = [vp, i]
        L.wema_cuda_batch_stage_times.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        L.wema_cuda_batch_stats.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                            C.POINTER(i)]
        L.wema_cuda_batch_read.argtypes = [vp, i, i, i, vp, sz]
        L.wema_cuda_batch_read.restype = C.c_long
        L.wema_cuda_server_create.argtypes = [i, sz, i, C.POINTER(vp)]
        L.wema_cuda_server_destroy.argtypes = [vp]
        L.wema_cuda_server_destroy.restype = None
        L.wema_cuda_server_open.argtypes = [vp, C.POINTER(Config), C.POINTER(i)]
        L.wema_cuda_server_submit.argtypes = [vp, i, vp, vp]
        L.wema_cuda_server_close.argtypes = [vp, i]
        L.wema_cuda_server_poll.argtypes = [vp, i, C.POINTER(SessionStatus)]
        L.wema_cuda_server_drain.argtypes = [vp, i]
        L.wema_cuda_server_hold.argtypes = [vp, i]
        L.wema_cuda_server_stats.argtypes = [vp, i, C.POINTER(ServeStats)]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().wema_cuda_last_error().decode()


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed: {last_error()}")


def make_config(width, height, fps=30.0, amp=120.0, f_low=0.5, f_high=None, window=32,
                edge_aware=True, bilateral=False, color=False, use_iir=True,
                threshold_form=THR_SINGLE, device=0, state_fp64=False, ring_fp16=False,
                planes_fp16=False) -> Config:
    c = Config()
    lib().wema_cuda_config_default(C.byref(c), int(width), int(height), float(fps))
    c.amp_factor = float(amp)
    c.f_low = float(f_low)
    if f_high is not None:
        c.f_high = float(f_high)
    c.temporal_window = int(window)
    c.edge_aware, c.bilateral_temp = int(bool(edge_aware)), int(bool(bilateral))
    c.color_mode, c.use_iir = int(bool(color)), int(bool(use_iir))
    c.threshold_form, c.device = int(threshold_form), int(device)
    c.iir_state_fp64 = int(bool(state_fp64))
    c.ring_fp16 = int(bool(ring_fp16))
    c.planes_fp16 = int(bool(planes_fp16))
    return c


def session_bytes(**kw) -> int:
    c = make_config(**kw)
    return int(lib().wema_cuda_session_bytes(C.byref(c)))


def _ptr(t) -> int:
    return t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data


class Session:
    """One video stream with device-resident state."""

    def __init__(self, inspect: bool = True, **kw):
        self.cfg = make_config(**kw)
        h = C.c_void_p()
        _check(lib().wema_cuda_session_create(C.byref(self.cfg), C.byref(h)), "session create")
        self.h = h
        _check(lib().wema_cuda_set_inspect(self.h, int(bool(inspect))), "set_inspect")
        self.w, self.hgt = self.cfg.width, self.cfg.height
        self.channels = 3 if self.cfg.color_mode else 1

    def process_u8(self, d_in, d_out, stream=None):
        s = stream.cuda_stream if stream is not None else None
        _check(lib().wema_cuda_process_u8(self.h, _ptr(d_in), _ptr(d_out), s), "process_u8")

    def process_u8_async(self, d_in, d_out, wait_event=None, done_event=None):
        """wait_event / done_event: torch.cuda.Event (or None)."""
        we = wait_event.cuda_event if wait_event is not None else None
        de = done_event.cuda_event if done_event is not None else None
        _check(lib().wema_cuda_process_u8_async(self.h, _ptr(d_in), _ptr(d_out), we, de),
               "process_u8_async")

    def process_f32(self, d_in, d_out_f32=None, d_out_u8=None, stream=None):
        s = stream.cuda_stream if stream is not None else None
        _check(lib().wema_cuda_process_f32(
            self.h, _ptr(d_in), _ptr(d_out_f32) if d_out_f32 is not None else None,
            _ptr(d_out_u8) if d_out_u8 is not None else None, s), "process_f32")

    def process_host_u8(self, frame: np.ndarray) -> np.ndarray:
        frame = np.ascontiguousarray(frame, np.uint8)
        out = np.empty_like(frame)
        _check(lib().wema_cuda_process_host_u8(self.h, frame.ctypes.data, out.ctypes.data),
               "process_host_u8")
        return out

    def snapshot(self) -> np.ndarray:
        """The stream's whole state as host bytes (wema_cuda_session_snapshot)."""
        n = lib().wema_cuda_session_snapshot_bytes(self.h)
        buf = np.empty(n, np.uint8)
        _check(lib().wema_cuda_session_snapshot(self.h, buf.ctypes.data, n), "session_snapshot")
        return buf

    def restore(self, snap: np.ndarray):
        snap = np.ascontiguousarray(snap, np.uint8)
        _check(lib().wema_cuda_session_restore(self.h, snap.ctypes.data, snap.size), "session_restore")

    def sync(self):
        _check(lib().wema_cuda_session_sync(self.h), "sync")

    @property
    def frames_processed(self) -> int:
        return lib().wema_cuda_session_frames_processed(self.h)

    def read(self, what: int, channel: int = 0, cap: int | None = None) -> np.ndarray:
        if cap is None:
            cap = max(8 * self.w * self.hgt + 64, 64)
        buf = np.empty(cap, np.float32)
        n = lib().wema_cuda_session_read(self.h, what, channel, buf.ctypes.data, cap)
        if n < 0:
            raise RuntimeError(f"read failed: {last_error()}")
        return buf[:n].copy()

    STAGES = ("fwd_dwt_level0", "fwd_dwt_levels", "threshold", "temporal_amplify",
              "inv_dwt_levels", "inv_dwt_level0", "luma_transfer")

    def set_timing(self, enable: bool):
        _check(lib().wema_cuda_set_timing(self.h, int(bool(enable))), "set_timing")

    def stage_times(self):
        """-> (dict stage -> total ms, frames timed)"""
        t = (C.c_double * len(self.STAGES))()
        n = C.c_longlong()
        _check(lib().wema_cuda_stage_times(self.h, t, C.byref(n)), "stage_times")
        return dict(zip(self.STAGES, list(t))), n.value

    def launches(self) -> int:
        """kernel launches issued by this session so far"""
        n = C.c_longlong()
        _check(lib().wema_cuda_session_launches(self.h, C.byref(n)), "session_launches")
        return n.value

    def close(self):
        if getattr(self, "h", None):
            lib().wema_cuda_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def threshold_flat(d_x, threshold_form=THR_SINGLE, stream=None):
    """Exact reference threshold of a flat device float32 tensor -> (thr, sum)."""
    import torch
    out = torch.empty(2, dtype=torch.float32, device=d_x.device)
    s = stream.cuda_stream if stream is not None else None
    _check(lib().wema_cuda_threshold_flat(d_x.data_ptr(), d_x.numel(), threshold_form,
                                          out.data_ptr(), out.data_ptr() + 4, s), "threshold")
    torch.cuda.synchronize()
    v = out.cpu().numpy()
    return np.float32(v[0]), np.float32(v[1])


def threshold_flat_noalloc(d_x, threshold_form=THR_SINGLE, stream=None):
    """As threshold_flat, through the entry point that allocates nothing
    (scratch in a fixed device array inside the library) -> (thr, sum)."""
    import torch
    out = torch.empty(2, dtype=torch.float32, device=d_x.device)
    s = stream.cuda_stream if stream is not None else None
    _check(lib().wema_cuda_threshold_flat_noalloc(d_x.data_ptr(), d_x.numel(), threshold_form,
                                                  out.data_ptr(), out.data_ptr() + 4, s),
           "threshold (no-alloc)")
    torch.cuda.synchronize()
    v = out.cpu().numpy()
    return np.float32(v[0]), np.float32(v[1])


def batch_stream_bytes(**kw) -> int:
    """Device bytes one batched stream of this config holds (its admission cost)."""
    c = make_config(**kw)
    return int(lib().wema_cuda_batch_stream_bytes(C.byref(c)))


class Batch:
    """Many streams advanced one frame per tick, one launch per kernel type
    over all of them (wema_cuda_batch_*)."""

    def __init__(self, device=0, max_streams=64):
        self.h = C.c_void_p()
        self.device = device
        _check(lib().wema_cuda_batch_create(int(device), int(max_streams), C.byref(self.h)),
               "batch_create")
        self.streams = {}     # id -> (width, height, channels)

    def add(self, width, height, **kw) -> int:
        c = make_config(width, height, device=self.device, **kw)
        sid = C.c_int()
        _check(lib().wema_cuda_batch_add(self.h, C.byref(c), C.byref(sid)), "batch_add")
        self.streams[sid.value] = (width, height, 3 if kw.get("color") else 1)
        return sid.value

    def remove(self, sid: int):
        _check(lib().wema_cuda_batch_remove(self.h, int(sid)), "batch_remove")
        self.streams.pop(sid, None)

    def tick(self, ids, inputs, outputs, wait_event=None, done_event=None):
        n = len(ids)
        ia = (C.c_int * n)(*ids)
        pin = (C.c_void_p * n)(*[_ptr(t) for t in inputs])
        pout = (C.c_void_p * n)(*[_ptr(t) for t in outputs])
        w = C.c_void_p(wait_event.cuda_event) if wait_event is not None else None
        d = C.c_void_p(done_event.cuda_event) if done_event is not None else None
        _check(lib().wema_cuda_batch_tick(self.h, ia, pin, pout, n, w, d), "batch_tick")

    def snapshot(self, sid: int) -> np.ndarray:
        n = lib().wema_cuda_batch_snapshot_bytes(self.h, int(sid))
        buf = np.empty(n, np.uint8)
        _check(lib().wema_cuda_batch_snapshot(self.h, int(sid), buf.ctypes.data, n), "batch_snapshot")
        return buf

    def restore(self, sid: int, snap: np.ndarray):
        snap = np.ascontiguousarray(snap, np.uint8)
        _check(lib().wema_cuda_batch_restore(self.h, int(sid), snap.ctypes.data, snap.size), "batch_restore")

    def sync(self):
        _check(lib().wema_cuda_batch_sync(self.h), "batch_sync")

    def tick_host(self, ids, inputs, outputs, wait_event=None, done_event=None):
        """One tick with host frames (numpy arrays or pinned CPU tensors)."""
        n = len(ids)
        ia = (C.c_int * n)(*ids)
        pin = (C.c_void_p * n)(*[_ptr(t) for t in inputs])
        pout = (C.c_void_p * n)(*[_ptr(t) for t in outputs])
        w = C.c_void_p(wait_event.cuda_event) if wait_event is not None else None
        d = C.c_void_p(done_event.cuda_event) if done_event is not None else None
        _check(lib().wema_cuda_batch_tick_host(self.h, ia, pin, pout, n, w, d), "batch_tick_host")

    def set_graphs(self, enable: bool):
        _check(lib().wema_cuda_batch_set_graphs(self.h, int(bool(enable))), "set_graphs")

    def set_groups(self, groups: int):
        _check(lib().wema_cuda_batch_set_groups(self.h, int(groups)), "set_groups")

    def set_host_overlap(self, enable: bool):
        _check(lib().wema_cuda_batch_set_host_overlap(self.h, int(bool(enable))), "set_host_overlap")

    def set_timing(self, enable: bool):
        _check(lib().wema_cuda_batch_set_timing(self.h, int(bool(enable))), "batch_set_timing")

    def stage_times(self):
        """-> (dict stage -> total ms over the timed ticks, ticks timed)"""
        t = (C.c_double * len(Session.STAGES))()
        n = C.c_longlong()
        _check(lib().wema_cuda_batch_stage_times(self.h, t, C.byref(n)), "batch_stage_times")
        return dict(zip(Session.STAGES, list(t))), n.value

    def stats(self):
        t, l, n = C.c_longlong(), C.c_longlong(), C.c_int()
        _check(lib().wema_cuda_batch_stats(self.h, C.byref(t), C.byref(l), C.byref(n)), "batch_stats")
        return {"ticks": t.value, "launches": l.value, "live": n.value}

    def threshold(self, sid: int, channel=0) -> float:
        f = C.c_float()
        rc = lib().wema_cuda_batch_read(self.h, int(sid), READ_THRESHOLD, int(channel),
                                        C.byref(f), 4)
        if rc < 0:
            raise RuntimeError(f"batch_read failed: {last_error()}")
        return f.value

    def close(self):
        if getattr(self, "h", None):
            lib().wema_cuda_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The served request loop (wema_cuda_server_*): sessions admitted against
    a device-memory budget, frames batched continuously by a native
    dispatcher thread."""

    def __init__(self, device=0, budget_bytes=150 * 10**9, max_streams=256):
        self.h = C.c_void_p()
        self.device = device
        _check(lib().wema_cuda_server_create(int(device), int(budget_bytes), int(max_streams),
                                             C.byref(self.h)), "server_create")

    def open(self, width, height, **kw) -> int:
        c = make_config(width, height, device=self.device, **kw)
        sid = C.c_int()
        _check(lib().wema_cuda_server_open(self.h, C.byref(c), C.byref(sid)), "server_open")
        return sid.value

    def submit(self, sid, d_in, d_out) -> int:
        """0 accepted, 1 refused (session queued), 2 refused (8 pending)."""
        rc = lib().wema_cuda_server_submit(self.h, int(sid), _ptr(d_in), _ptr(d_out))
        if rc < 0:
            raise RuntimeError(f"server_submit failed: {last_error()}")
        return rc

    def close_session(self, sid):
        _check(lib().wema_cuda_server_close(self.h, int(sid)), "server_close")

    def poll(self, sid) -> dict:
        st = SessionStatus()
        _check(lib().wema_cuda_server_poll(self.h, int(sid), C.byref(st)), "server_poll")
        return {k: getattr(st, k) for k, _ in SessionStatus._fields_}

    def hold(self, on=True):
        _check(lib().wema_cuda_server_hold(self.h, int(bool(on))), "server_hold")

    def drain(self, timeout_ms=60000):
        _check(lib().wema_cuda_server_drain(self.h, int(timeout_ms)), "server_drain")

    def stats(self, reset=False) -> dict:
        st = ServeStats()
        _check(lib().wema_cuda_server_stats(self.h, int(bool(reset)), C.byref(st)), "server_stats")
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}

    def close(self):
        if self.h:
            lib().wema_cuda_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(device=0):
    """Times the filter step at 2 / 4 / 8 positions per thread and keeps the
    fastest for the device -> (positions, report)."""
    buf = C.create_string_buffer(1024)
    u = lib().wema_cuda_autotune(int(device), buf, 1024)
    if u < 0:
        raise RuntimeError(f"autotune failed: {last_error()}")
    return u, buf.value.decode()


def set_iir_positions(device, positions):
    _check(lib().wema_cuda_set_iir_positions(int(device), int(positions)), "set_iir_positions")


def iir_positions(device=0) -> int:
    return lib().wema_cuda_get_iir_positions(int(device))


def set_guided_rows(device, rows):
    _check(lib().wema_cuda_set_guided_rows(int(device), int(rows)), "set_guided_rows")


def guided_rows(device=0) -> int:
    return lib().wema_cuda_get_guided_rows(int(device))


def set_dwt_variant(device, inverse, variant):
    _check(lib().wema_cuda_set_dwt_variant(int(device), int(bool(inverse)), int(variant)), "set_dwt_variant")


def dwt_variant(device=0, inverse=False) -> int:
    return lib().wema_cuda_get_dwt_variant(int(device), int(bool(inverse)))
