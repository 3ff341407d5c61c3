"""Python binding of the at3r C ABI (include/at3r.h) and a mirror of the
reference's reconstruction entry points.

    vol = CDoWbpRecon().DoIt(tilt_series, align_param, vol_z)
    vol = CDoSartRecon().DoIt(tilt_series, align_param, start_tilt, num_tilts, vol_z, iterations, subsets)

follow ``MAR::CDoWbpRecon::DoIt`` / ``MAR::CDoSartRecon::DoIt``
(AreTomo/Recon/CReconInc.h:259-306): the tilt series is read, not modified;
the returned volume holds one XZ slice per y with z flipped, shape
(ny, vol_z, nx & ~1).  Errors raise ``ReconError`` instead of aborting.

All computation runs in libat3r.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import load_library

WBP, SART = 0, 1
STORE_F32, STORE_F16, STORE_BF16 = 0, 1, 2
C2R_MATCH_CUFFT, C2R_HERMITIAN, C2R_PACKED = 0, 1, 2


class ReconError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"at3r status {status}: {message}")
        self.status = status


class Geom(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("n_tilts", ctypes.c_int),
        ("tilts_deg", ctypes.POINTER(ctypes.c_float)),
        ("vol_z", ctypes.c_int),
        ("method", ctypes.c_int),
        ("start_tilt", ctypes.c_int), ("num_tilts", ctypes.c_int),
        ("iterations", ctypes.c_int), ("subsets", ctypes.c_int),
        ("relax", ctypes.c_float),
        ("storage", ctypes.c_int),
        ("c2r", ctypes.c_int),
        ("slab_slices", ctypes.c_int),
        ("compute_rfactor", ctypes.c_int),
        ("fill_seed", ctypes.c_ulonglong),
    ]


class StackGeom(ctypes.Structure):
    """at3r_stack_geom (include/at3r.h)."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("n_tilts", ctypes.c_int), ("correct", ctypes.c_int),
                ("shifts", ctypes.c_void_p), ("tilt_axes_deg", ctypes.c_void_p), ("size_axis_deg", ctypes.c_float),
                ("num_patches", ctypes.c_int), ("local_params", ctypes.c_void_p), ("rand_fill", ctypes.c_int),
                ("seed", ctypes.c_ulonglong), ("bin", ctypes.c_float)]


class ThicknessResult(ctypes.Structure):
    """at3r_thickness (include/at3r.h)."""
    _fields_ = [("binning", ctypes.c_float), ("binned_xy", ctypes.c_int * 2), ("vol_z", ctypes.c_int),
                ("n_profile", ctypes.c_int), ("edges", ctypes.c_int * 2), ("thickness", ctypes.c_int),
                ("offset_z", ctypes.c_int)]


_EXPORTS = {
    "at3r_geom_init": (None, [ctypes.POINTER(Geom), ctypes.c_int]),
    "at3r_plan_create": (ctypes.c_int, [ctypes.POINTER(Geom), ctypes.POINTER(ctypes.c_void_p)]),
    "at3r_plan_destroy": (None, [ctypes.c_void_p]),
    "at3r_run_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "at3r_run_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    "at3r_run_host_xyz": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p,
                                         ctypes.c_int, ctypes.c_void_p]),
    "at3r_volume_xyz": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    "at3r_get_rfactor": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    "at3r_plan_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "at3r_plan_last_launches": (ctypes.c_int64, [ctypes.c_void_p]),
    "at3r_plan_c2r": (ctypes.c_int, [ctypes.c_void_p]),
    "at3r_plan_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "at3r_plan_kernel_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                              ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "at3r_plan_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_int)]),
    "at3r_plan_slab": (ctypes.c_int, [ctypes.c_void_p]),
    "at3r_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "at3r_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "at3r_batch_destroy": (None, [ctypes.c_void_p]),
    "at3r_plan_estimate_bytes": (ctypes.c_size_t, [ctypes.POINTER(Geom)]),
    "at3r_server_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "at3r_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Geom), ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64)]),
    "at3r_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]),
    "at3r_server_in_use_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "at3r_server_destroy": (None, [ctypes.c_void_p]),
    "at3r_release_cached_memory": (None, []),
    "at3r_reproj_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p]),
    "at3r_reproj_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "at3r_reproj_host": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "at3r_stack_geom_init": (None, [ctypes.POINTER(StackGeom)]),
    "at3r_stack_create": (ctypes.c_int, [ctypes.POINTER(StackGeom), ctypes.POINTER(ctypes.c_void_p)]),
    "at3r_stack_destroy": (None, [ctypes.c_void_p]),
    "at3r_stack_sizes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "at3r_stack_c2r": (ctypes.c_int, [ctypes.c_void_p]),
    "at3r_stack_fill_table": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "at3r_stack_run_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "at3r_stack_run_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    "at3r_thickness_device": (ctypes.c_int, [ctypes.POINTER(StackGeom), ctypes.c_void_p, ctypes.c_float,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.POINTER(ThicknessResult), ctypes.c_void_p]),
    "at3r_thickness_host": (ctypes.c_int, [ctypes.POINTER(StackGeom), ctypes.c_void_p, ctypes.c_float,
                                           ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_int, ctypes.POINTER(ThicknessResult), ctypes.c_void_p]),
    "at3r_mrc_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_float]),
    "at3r_plan_flags_seen": (ctypes.c_int, [ctypes.c_void_p]),
    "at3r_plan_fill_table": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "at3r_batch_set_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "at3r_batch_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "at3r_status_str": (ctypes.c_char_p, [ctypes.c_int]),
    "at3r_last_error": (ctypes.c_char_p, []),
}


def lib() -> ctypes.CDLL:
    L = load_library("libat3r.so")
    if not getattr(L, "_at3r_typed", False):
        for name, (res, args) in _EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L._at3r_typed = True
    return L


def _check(rc: int) -> None:
    if rc != 0:
        L = lib()
        raise ReconError(rc, f"{L.at3r_status_str(rc).decode()}: {L.at3r_last_error().decode()}")


def make_geom(nx, ny, tilts_deg, vol_z, method=WBP, start_tilt=0, num_tilts=None, iterations=0, subsets=1,
              relax=0.0, storage=STORE_F32, c2r=C2R_MATCH_CUFFT, slab_slices=0, compute_rfactor=False,
              fill_seed=None):
    """Fills an at3r_geom; returns it with the tilt array it points into
    (which the caller keeps alive as long as the struct).  fill_seed: seed of
    SART's empty-voxel fill table; None keeps at3r_geom_init's time(0), as the
    reference seeds it."""
    tilts = np.ascontiguousarray(np.asarray(tilts_deg, dtype=np.float32))
    g = Geom()
    lib().at3r_geom_init(ctypes.byref(g), method)
    g.nx, g.ny, g.n_tilts = int(nx), int(ny), int(tilts.size)
    g.tilts_deg = tilts.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    g.vol_z = int(vol_z)
    g.start_tilt = int(start_tilt)
    g.num_tilts = int(tilts.size if num_tilts is None else num_tilts)
    g.iterations, g.subsets, g.relax = int(iterations), int(subsets), float(relax)
    g.storage, g.c2r, g.slab_slices = int(storage), int(c2r), int(slab_slices)
    g.compute_rfactor = int(bool(compute_rfactor))
    if fill_seed is not None:
        g.fill_seed = int(fill_seed)
    return g, tilts


class Plan:
    """One reconstruction plan (geometry, parameters and device workspace)."""

    def __init__(self, nx, ny, tilts_deg, vol_z, method=WBP, start_tilt=0, num_tilts=None, iterations=0,
                 subsets=1, relax=0.0, storage=STORE_F32, c2r=C2R_MATCH_CUFFT, slab_slices=0,
                 compute_rfactor=False, fill_seed=None):
        L = lib()
        g, self._tilts = make_geom(nx, ny, tilts_deg, vol_z, method, start_tilt, num_tilts, iterations, subsets,
                                   relax, storage, c2r, slab_slices, compute_rfactor, fill_seed)
        self.geom = g
        self.method = method
        self.iterations = int(iterations)
        self.nx, self.ny, self.vol_z = int(nx), int(ny), int(vol_z)
        self.Nx = self.nx & ~1
        h = ctypes.c_void_p()
        _check(L.at3r_plan_create(ctypes.byref(g), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().at3r_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def volume_shape(self):
        return (self.ny, self.vol_z, self.Nx)

    def run_device(self, proj_ptr: int, vol_ptr: int, stream: int = 0) -> None:
        """proj_ptr / vol_ptr: device addresses of float[T][ny][nx] / float[ny][Nz][Nx]."""
        _check(lib().at3r_run_device(self._h, ctypes.c_void_p(proj_ptr), ctypes.c_void_p(vol_ptr),
                                     ctypes.c_void_p(stream)))

    def run_host(self, frames, vol_frames, stream: int = 0) -> None:
        """frames: sequence of T host float32 arrays [ny][nx]; vol_frames: ny host
        float32 arrays [Nz][Nx], written in place."""
        T = len(frames)
        fin = (ctypes.c_void_p * T)(*[f.ctypes.data for f in frames])
        fout = (ctypes.c_void_p * len(vol_frames))(*[v.ctypes.data for v in vol_frames])
        _check(lib().at3r_run_host(self._h, fin, fout, ctypes.c_void_p(stream)))

    def run_host_xyz(self, frames, out: np.ndarray | None = None, flip: bool = True, stream: int = 0) -> np.ndarray:
        """Reconstructs and returns the volume as XY frames [Nz][ny][Nx], as
        CTiltSeries::FlipVol(flip) gives them (flip: frames in z order)."""
        T = len(frames)
        if out is None:
            out = np.empty((self.vol_z, self.ny, self.Nx), np.float32)
        if out.shape != (self.vol_z, self.ny, self.Nx) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array [vol_z][ny][Nx]")
        fin = (ctypes.c_void_p * T)(*[f.ctypes.data for f in frames])
        _check(lib().at3r_run_host_xyz(self._h, fin, ctypes.c_void_p(out.ctypes.data), int(bool(flip)),
                                       ctypes.c_void_p(stream)))
        return out

    def rfactor(self) -> np.ndarray:
        """Per iteration (sum|raw - fp|, sum|raw|) of the last run."""
        out = np.zeros(2 * max(self.iterations, 1), np.float64)
        _check(lib().at3r_get_rfactor(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size))
        return out[: 2 * self.iterations].reshape(self.iterations, 2)

    @property
    def workspace_bytes(self) -> int:
        return int(lib().at3r_plan_workspace_bytes(self._h))

    @property
    def last_launches(self) -> int:
        return int(lib().at3r_plan_last_launches(self._h))

    @property
    def c2r(self) -> int:
        return int(lib().at3r_plan_c2r(self._h))

    def flags_seen(self) -> int:
        """Bits of what the last run met (at3r_plan_flags_seen): 1 empty SART
        voxels (filled), 2 staged projections near the missing-value test, 4
        the residual near it, 8 a fill chain took the slice mean."""
        v = int(lib().at3r_plan_flags_seen(self._h))
        if v < 0:
            _check(2)
        return v

    def fill_table(self) -> np.ndarray:
        """The SART fill's random table, Nx * vol_z int32 (reference voxel order)."""
        out = np.empty(self.Nx * self.vol_z, np.int32)
        _check(lib().at3r_plan_fill_table(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def autotune(self, proj_ptr: int, vol_ptr: int, stream: int = 0) -> int:
        """Times candidate slab sizes on the given device buffers (overwritten)
        and keeps the fastest; returns it."""
        chosen = ctypes.c_int()
        _check(lib().at3r_plan_autotune(self._h, ctypes.c_void_p(proj_ptr), ctypes.c_void_p(vol_ptr),
                                        ctypes.c_void_p(stream), ctypes.byref(chosen)))
        return chosen.value

    @property
    def slab(self) -> int:
        return int(lib().at3r_plan_slab(self._h))

    def set_timing(self, enable: bool) -> None:
        _check(lib().at3r_plan_set_timing(self._h, int(bool(enable))))

    def kernel_stats(self) -> dict:
        """Per kernel kind of the last run: launches, device ms (timing on),
        algorithmic bytes, work units."""
        L = lib()
        out = {}
        n = L.at3r_plan_kernel_stats(self._h, 0, None, None, None, None, None)
        for k in range(n):
            name = ctypes.c_char_p()
            la = ctypes.c_int64()
            ms, by, un = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
            L.at3r_plan_kernel_stats(self._h, k, ctypes.byref(name), ctypes.byref(la), ctypes.byref(ms),
                                     ctypes.byref(by), ctypes.byref(un))
            if la.value:
                out[name.value.decode()] = dict(launches=la.value, ms=ms.value, bytes=by.value, units=un.value)
        return out


class Batch:
    """Several plans over device-resident series, captured into one CUDA graph
    and replayed as one launch.  WBP plans of one storage type run as waves of
    persistent stage kernels across all series (at3r_batch_create); other
    mixes capture each plan's launches on parallel branches."""

    MODES = {"auto": 0, "branches": 1, "waves": 2}

    def __init__(self, plans, proj_ptrs, vol_ptrs, branches: int = 4, mode: str = "auto"):
        n = len(plans)
        P = ctypes.c_void_p * n
        self._plans = list(plans)   # keep the plans alive
        h = ctypes.c_void_p()
        _check(lib().at3r_batch_create(P(*[p._h.value for p in plans]), P(*proj_ptrs), P(*vol_ptrs), n,
                                       int(branches), ctypes.byref(h)))
        self._h = h
        if mode != "auto":
            _check(lib().at3r_batch_set_mode(self._h, self.MODES[mode]))

    @property
    def mode(self):
        """("branches" | "waves" | None before the first run, ms of the wave
        form, ms of the branch form) — the timings when the first run chose."""
        mw, mb = ctypes.c_float(), ctypes.c_float()
        m = int(lib().at3r_batch_mode(self._h, ctypes.byref(mw), ctypes.byref(mb)))
        return {0: None, 1: "branches", 2: "waves"}[m], mw.value, mb.value

    def run(self, stream: int = 0) -> None:
        _check(lib().at3r_batch_run(self._h, ctypes.c_void_p(stream)))

    def close(self):
        if getattr(self, "_h", None):
            lib().at3r_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_bytes(nx, ny, tilts_deg, vol_z, **kw) -> int:
    """Device bytes a plan plus one host-path run hold, by estimate (no GPU)."""
    g, _t = make_geom(nx, ny, tilts_deg, vol_z, **kw)
    return int(lib().at3r_plan_estimate_bytes(ctypes.byref(g)))


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_inflight", ctypes.c_int)]


class Server:
    """Serving loop on the current device (at3r_server_*): tilt series are
    submitted as they arrive; a request is admitted when its device bytes
    (plan workspace, its projections held on the device, two volume slabs)
    fit the HBM budget and fewer than max_inflight requests are active, and
    the slabs of the active requests interleave on the device (continuous
    batching at y-slab granularity), each finished slab streamed to host."""

    def __init__(self, hbm_budget_bytes: int = 0, max_inflight: int = 4):
        o = ServerOpts(int(hbm_budget_bytes), int(max_inflight))
        h = ctypes.c_void_p()
        _check(lib().at3r_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, frames: np.ndarray, tilts_deg, vol_z: int, out: np.ndarray | None = None,
               out_frames=None, **kw) -> int:
        """frames: host float32 [T][ny][nx] (pinned memory overlaps best);
        returns a request id.  The volume lands in `out` (allocated if None),
        which wait() returns; or, with out_frames, in those ny frames of
        [vol_z][nx & ~1] float32 (they may repeat: a ring that keeps only the
        last rows written, for timing series whose volume exceeds host memory)."""
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        T, ny, nx = frames.shape
        g, tilts = make_geom(nx, ny, tilts_deg, vol_z, **kw)
        if out_frames is not None:
            if len(out_frames) != ny:
                raise ValueError("out_frames needs one frame per row")
            fout = (ctypes.c_void_p * ny)(*[f.ctypes.data for f in out_frames])
            out = out_frames
        else:
            if out is None:
                out = np.empty((ny, int(vol_z), nx & ~1), np.float32)
            fout = (ctypes.c_void_p * ny)(*[out[y].ctypes.data for y in range(ny)])
        fin = (ctypes.c_void_p * T)(*[frames[t].ctypes.data for t in range(T)])
        rid = ctypes.c_int64()
        _check(lib().at3r_server_submit(self._h, ctypes.byref(g), fin, fout, ctypes.byref(rid)))
        self._keep[rid.value] = (frames, out, tilts, fin, fout)
        return rid.value

    def wait(self, rid: int):
        """Blocks until the request is done; returns (volume, latency_s, queued_s)."""
        lat, q = ctypes.c_double(), ctypes.c_double()
        try:
            _check(lib().at3r_server_wait(self._h, int(rid), ctypes.byref(lat), ctypes.byref(q)))
        finally:
            kept = self._keep.pop(int(rid), None)
        return kept[1], lat.value, q.value

    @property
    def in_use_bytes(self) -> int:
        return int(lib().at3r_server_in_use_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().at3r_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- reference-shaped entry points -----------------------------------------

@dataclass
class TiltSeries:
    """The aligned tilt series: frames[T][ny][nx] float32 (MD::CTiltSeries)."""
    frames: np.ndarray

    @property
    def stk_size(self):
        t, ny, nx = self.frames.shape
        return (nx, ny, t)


@dataclass
class AlignParam:
    """MAM::CAlignParam: per-tilt angles in degrees with the alpha offset
    folded in (GetTilts), global shifts in pixels (GetShift) and tilt axes in
    degrees (GetTiltAxis)."""
    tilts: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    shifts: np.ndarray | None = None       # [T][2]
    tilt_axes: np.ndarray | None = None    # [T]

    def GetTilts(self, copy: bool = False):
        return self.tilts.copy() if copy else self.tilts

    def GetShift(self, i: int):
        return (0.0, 0.0) if self.shifts is None else tuple(float(v) for v in self.shifts[i])

    def GetTiltAxis(self, i: int) -> float:
        return 0.0 if self.tilt_axes is None else float(self.tilt_axes[i])


@dataclass
class LocalAlignParam:
    """MAM::CLocalAlignParam: per tilt, five rows of num_patches values
    (patch centre x, centre y, shift x, shift y, good flag), [T][5][P]."""
    params: np.ndarray

    @property
    def m_iNumPatches(self) -> int:
        return int(self.params.shape[2])


def _host_run(plan: Plan, frames: np.ndarray) -> np.ndarray:
    frames = np.ascontiguousarray(frames, dtype=np.float32)
    vol = np.empty(plan.volume_shape, np.float32)
    plan.run_host([frames[t] for t in range(frames.shape[0])], [vol[y] for y in range(vol.shape[0])])
    return vol


class CDoWbpRecon:
    """MAR::CDoWbpRecon (AreTomo/Recon/CDoWbpRecon.cpp:28-47)."""

    def __init__(self, **options):
        self.options = options

    def DoIt(self, tilt_series: TiltSeries, align_param: AlignParam, vol_z: int) -> np.ndarray:
        nx, ny, nt = tilt_series.stk_size
        plan = Plan(nx, ny, align_param.GetTilts(False)[:nt], vol_z, method=WBP, **self.options)
        try:
            return _host_run(plan, tilt_series.frames)
        finally:
            plan.close()


class CDoSartRecon:
    """MAR::CDoSartRecon (AreTomo/Recon/CDoSartRecon.cpp:30-57)."""

    def __init__(self, **options):
        self.options = options

    def DoIt(self, tilt_series: TiltSeries, align_param: AlignParam, start_tilt: int, num_tilts: int, vol_z: int,
             iterations: int, subsets: int) -> np.ndarray:
        nx, ny, nt = tilt_series.stk_size
        plan = Plan(nx, ny, align_param.GetTilts(False)[:nt], vol_z, method=SART, start_tilt=start_tilt,
                    num_tilts=num_tilts, iterations=iterations, subsets=subsets, **self.options)
        try:
            return _host_run(plan, tilt_series.frames)
        finally:
            plan.close()


def volume_xyz(vol, flip: bool = True, out=None, stream=None):
    """Device transpose of a torch CUDA volume vol[ny][Nz][Nx] (XZ frames) to
    XY frames [Nz][ny][Nx], as CTiltSeries::FlipVol(flip)."""
    import torch
    if not (vol.is_cuda and vol.dtype == torch.float32 and vol.is_contiguous() and vol.dim() == 3):
        raise ValueError("vol must be a contiguous float32 CUDA tensor [ny][Nz][Nx]")
    ny, nz, nx = vol.shape
    if out is None:
        out = torch.empty((nz, ny, nx), device=vol.device, dtype=torch.float32)
    s = stream if stream is not None else torch.cuda.current_stream(vol.device)
    _check(lib().at3r_volume_xyz(ctypes.c_void_p(vol.data_ptr()), nx, ny, nz, int(bool(flip)),
                                 ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream)))
    return out


class CCalcReproj:
    """Mirror of ProjAlign::CCalcReproj (AreTomo/ProjAlign/CCalcReproj.cpp):
    Setup(stack size, vol_z), then DoIt(frames, tilts, skip, proj_idx) returns
    the re-projection of tilt proj_idx, [ny][nx] float32 (-1e30 where a ray
    covers under 80 %).  skip: per-tilt flags as the caller keeps them (the
    caller marks proj_idx itself, as CProjAlignMain::mCalcReproj does)."""

    def Setup(self, tomo_stk_size, vol_z: int, nth_gpu: int = 0):
        self.nx, self.ny, self.nt = (int(v) for v in tomo_stk_size)
        self.vol_z = int(vol_z)

    def DoIt(self, frames, tilts, skip, proj_idx: int, out: np.ndarray | None = None) -> np.ndarray:
        tilts = np.ascontiguousarray(tilts, np.float32)
        sk = None if skip is None else np.ascontiguousarray(skip, np.uint8)
        if out is None:
            out = np.empty((self.ny, self.nx), np.float32)
        fr = (ctypes.c_void_p * self.nt)(*[np.ascontiguousarray(f, np.float32).ctypes.data if f is not None else None
                                           for f in frames])
        self._keep = frames
        _check(lib().at3r_reproj_host(fr, self.nx, self.ny, self.nt, tilts.ctypes.data,
                                      sk.ctypes.data if sk is not None else None, int(proj_idx), self.vol_z,
                                      out.ctypes.data, None))
        return out


def reproj_range(tilts, proj_idx: int, skip=None):
    """The tilt range [first, last] CCalcReproj::mFindProjRange picks."""
    tilts = np.ascontiguousarray(tilts, np.float32)
    sk = None if skip is None else np.ascontiguousarray(skip, np.uint8)
    rng = np.zeros(2, np.int32)
    _check(lib().at3r_reproj_range(tilts.ctypes.data, sk.ctypes.data if sk is not None else None, tilts.size,
                                   int(proj_idx), rng.ctypes.data))
    return int(rng[0]), int(rng[1])


def reproj_device(proj, tilts, proj_idx: int, vol_z: int, skip=None, out=None, stream=None):
    """Re-projection of tilt proj_idx from a torch CUDA tensor proj[T][ny][nx]."""
    import torch
    if not (proj.is_cuda and proj.dtype == torch.float32 and proj.is_contiguous()):
        raise ValueError("proj must be a contiguous float32 CUDA tensor")
    T, ny, nx = proj.shape
    tilts = np.ascontiguousarray(tilts, np.float32)
    sk = None if skip is None else np.ascontiguousarray(skip, np.uint8)
    if out is None:
        out = torch.empty((ny, nx), device=proj.device, dtype=torch.float32)
    s = stream if stream is not None else torch.cuda.current_stream(proj.device)
    _check(lib().at3r_reproj_device(ctypes.c_void_p(proj.data_ptr()), nx, ny, T, tilts.ctypes.data,
                                    sk.ctypes.data if sk is not None else None, int(proj_idx), int(vol_z),
                                    ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream)))
    return out


def reconstruct_device(proj, tilts, vol_z, method=WBP, out=None, stream=None, **kw):
    """Device-resident reconstruction of a torch CUDA tensor proj[T][ny][nx]
    (float32, contiguous).  Returns (or fills) vol[ny][vol_z][nx & ~1]."""
    import torch
    if not (proj.is_cuda and proj.dtype == torch.float32 and proj.is_contiguous()):
        raise ValueError("proj must be a contiguous float32 CUDA tensor")
    T, ny, nx = proj.shape
    plan = Plan(nx, ny, tilts, vol_z, method=method, **kw)
    if out is None:
        out = torch.empty(plan.volume_shape, device=proj.device, dtype=torch.float32)
    s = stream if stream is not None else torch.cuda.current_stream(proj.device)
    plan.run_device(proj.data_ptr(), out.data_ptr(), s.cuda_stream)
    return out, plan


# --- input stage and thickness measurement -----------------------------------

def _stack_geom(nx, ny, n_tilts, correct=True, shifts=None, tilt_axes=None, size_axis=0.0, local_params=None,
                rand_fill=True, seed=None, bin=1.0):
    """at3r_stack_geom plus the arrays it points at (kept alive by the caller)."""
    g = StackGeom()
    lib().at3r_stack_geom_init(ctypes.byref(g))
    g.nx, g.ny, g.n_tilts = int(nx), int(ny), int(n_tilts)
    g.correct = int(bool(correct))
    keep = []
    if shifts is not None:
        a = np.ascontiguousarray(shifts, np.float32).reshape(n_tilts, 2)
        keep.append(a)
        g.shifts = a.ctypes.data
    if tilt_axes is not None:
        a = np.ascontiguousarray(tilt_axes, np.float32).reshape(n_tilts)
        keep.append(a)
        g.tilt_axes_deg = a.ctypes.data
    g.size_axis_deg = float(size_axis)
    if local_params is not None:
        a = np.ascontiguousarray(local_params, np.float32)
        if a.ndim != 3 or a.shape[0] != n_tilts or a.shape[1] != 5:
            raise ValueError("local_params must be [n_tilts][5][num_patches]")
        keep.append(a)
        g.num_patches = int(a.shape[2])
        g.local_params = a.ctypes.data
    g.rand_fill = int(bool(rand_fill))
    g.seed = int(time.time()) if seed is None else int(seed)
    g.bin = float(bin)
    return g, keep


class Stack:
    """An at3r_stack: aligned (shift / rotation / local patches + random fill)
    and Fourier-binned tilt frames.  Arguments as at3r_stack_geom; seed None
    seeds the fill's table with the time, as the reference does."""

    def __init__(self, nx, ny, n_tilts, **kw):
        g, keep = _stack_geom(nx, ny, n_tilts, **kw)
        h = ctypes.c_void_p()
        _check(lib().at3r_stack_create(ctypes.byref(g), ctypes.byref(h)))
        self._h = h
        self.n_tilts = int(n_tilts)
        self.raw_shape = (int(n_tilts), int(ny), int(nx))
        a, b = (ctypes.c_int * 2)(), (ctypes.c_int * 2)()
        _check(lib().at3r_stack_sizes(h, a, b))
        self.aligned_xy = (a[0], a[1])
        self.binned_xy = (b[0], b[1])
        self.seed = int(g.seed)

    @property
    def binned_shape(self):
        return (self.n_tilts, self.binned_xy[1], self.binned_xy[0])

    def run_device(self, raw_ptr: int, out_ptr: int, stream: int = 0) -> None:
        _check(lib().at3r_stack_run_device(self._h, ctypes.c_void_p(raw_ptr), ctypes.c_void_p(out_ptr),
                                           ctypes.c_void_p(stream)))

    def run_host(self, frames, out=None, stream: int = 0) -> np.ndarray:
        frames = [np.ascontiguousarray(f, np.float32) for f in frames]
        if out is None:
            out = np.empty(self.binned_shape, np.float32)
        P = ctypes.c_void_p * self.n_tilts
        _check(lib().at3r_stack_run_host(self._h, P(*[f.ctypes.data for f in frames]),
                                         P(*[out[t].ctypes.data for t in range(self.n_tilts)]),
                                         ctypes.c_void_p(stream)))
        return out

    @property
    def c2r(self) -> int:
        """C2R convention of the binning (C2R_HERMITIAN or C2R_PACKED)."""
        return int(lib().at3r_stack_c2r(self._h))

    def fill_table(self) -> np.ndarray:
        """The random table of the fill (W * ay entries, W = ax rounded down to even)."""
        W = self.aligned_xy[0] & ~1
        out = np.empty(W * self.aligned_xy[1], np.int32)
        _check(lib().at3r_stack_fill_table(self._h, out.ctypes.data, out.size))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().at3r_stack_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CCorrTomoStack:
    """Mirror of MAC::CCorrTomoStack (AreTomo/Correct/CCorrTomoStack.cpp:66-222)
    set up with Fourier cropping: Set0(series) .. Set4, DoIt, GetCorrectedStack.
    Set0 takes the tilt series whose size the reference reads from its series
    package; DoIt takes the alignment (and local alignment, if Set1 was given
    patches) the reference reads from its singletons.  Real-space binning
    (Set2 with bFourierCrop = false) and the R-weighting of Set3 are not
    part of this path."""

    def Set0(self, tilt_series: "TiltSeries"):
        self._series = tilt_series
        self._corrected = None

    def Set1(self, num_patches: int, tilt_axis: float):
        self._patches, self._size_axis = int(num_patches), float(tilt_axis)

    def Set2(self, out_bin: float, fourier_crop: bool = True, rand_fill: bool = True):
        if not fourier_crop:
            raise NotImplementedError("real-space binning (GBinImage2D) is not part of this path")
        self._bin = float(out_bin)
        self._rand_fill = True   # CCorrTomoStack::Set2 forces it with Fourier cropping

    def Set3(self, shift_only: bool, corr_int: bool, rweight: bool):
        if rweight:
            raise NotImplementedError("the R-weighted corrected stack is not part of this path")
        self._shift_only = bool(shift_only)

    def Set4(self, for_recon: bool):
        self._for_recon = bool(for_recon)

    def DoIt(self, align_param: "AlignParam", local_param: "LocalAlignParam | None" = None, seed=None):
        nx, ny, nt = self._series.stk_size
        axes = None
        if not self._shift_only:
            axes = np.asarray([align_param.GetTiltAxis(i) for i in range(nt)], np.float32)
        local = None
        if self._patches > 0 and local_param is not None:
            local = local_param.params
        st = Stack(nx, ny, nt, shifts=np.asarray([align_param.GetShift(i) for i in range(nt)], np.float32),
                   tilt_axes=axes, size_axis=self._size_axis, local_params=local, rand_fill=self._rand_fill,
                   seed=seed, bin=self._bin)
        try:
            out = st.run_host([self._series.frames[t] for t in range(nt)])
            self._aligned_xy, self._binned_xy = st.aligned_xy, st.binned_xy
        finally:
            st.close()
        self._corrected = TiltSeries(out)
        return self._corrected

    def GetCorrectedStack(self, clean: bool = False) -> "TiltSeries":
        out = self._corrected
        if clean:
            self._corrected = None
        return out

    def GetBinning(self):
        """m_afBinning: aligned / binned size per dimension."""
        return (np.float32(self._aligned_xy[0]) / np.float32(self._binned_xy[0]),
                np.float32(self._aligned_xy[1]) / np.float32(self._binned_xy[1]))


class CBinStack:
    """Mirror of MAC::CBinStack::DoFFT (AreTomo/Correct/CBinStack.cpp:61-106)."""

    @staticmethod
    def DoFFT(tilt_series: "TiltSeries", bin: float) -> "TiltSeries":
        nx, ny, nt = tilt_series.stk_size
        st = Stack(nx, ny, nt, correct=False, rand_fill=False, seed=0, bin=bin)
        try:
            return TiltSeries(st.run_host([tilt_series.frames[t] for t in range(nt)]))
        finally:
            st.close()


def thickness_pixel_size(pix_size: float, nx: int, ny: int, tilt_axis: float, binned_y: int, binning) -> np.float32:
    """The pixel size CCalcVolThick's edges are scaled by in Angstrom: the raw
    pixel size times CCorrTomoStack's y binning (aligned y / binned y, the
    aligned size as CCorrectUtil::CalcAlignedSize gives it), over the
    binning (CCorrTomoStack.cpp:129-131, 180; CCalcVolThick.cpp:73)."""
    aligned_y = nx if abs(np.sin(float(tilt_axis) * 3.14 / 180.0)) > 0.707 else ny
    bin_y = np.float32(aligned_y) / np.float32(binned_y)
    return np.float32(np.float32(np.float32(pix_size) * bin_y) / np.float32(binning))


class CCalcVolThick:
    """Mirror of MAR::CCalcVolThick (AreTomo/Recon/CCalcVolThick.cpp:47-110):
    DoIt(series, alignment, pixel size) aligns and bins the series by
    max(20 / pixel size, 20), reconstructs it by WBP, measures the standard
    deviation of every z plane and finds the sample's edges.  The tilt axis of
    tilt 0 sizes the aligned frame (Set1 of the reference's call)."""

    def DoIt(self, tilt_series: "TiltSeries", align_param: "AlignParam", pix_size: float, seed=None):
        nx, ny, nt = tilt_series.stk_size
        axes = np.asarray([align_param.GetTiltAxis(i) for i in range(nt)], np.float32)
        g, keep = _stack_geom(nx, ny, nt, shifts=np.asarray([align_param.GetShift(i) for i in range(nt)], np.float32),
                              tilt_axes=axes, size_axis=float(axes[0]), rand_fill=True, seed=seed)
        self.seed = int(g.seed)
        tilts = np.ascontiguousarray(align_param.GetTilts(False)[:nt], np.float32)
        frames = [np.ascontiguousarray(tilt_series.frames[t], np.float32) for t in range(nt)]
        cap = 4096
        prof, prof_s = np.zeros(cap, np.float32), np.zeros(cap, np.float32)
        r = ThicknessResult()
        P = ctypes.c_void_p * nt
        _check(lib().at3r_thickness_host(ctypes.byref(g), tilts.ctypes.data, float(pix_size),
                                         P(*[f.ctypes.data for f in frames]), prof.ctypes.data, prof_s.ctypes.data,
                                         cap, ctypes.byref(r), None))
        self.result = r
        n = r.n_profile
        self.profile, self.profile_smoothed = prof[:n].copy(), prof_s[:n].copy()
        self.m_aiSampleEdges = (r.edges[0], r.edges[1])
        self.m_fBinning = np.float32(r.binning)
        self.m_fPixSize = thickness_pixel_size(pix_size, nx, ny, float(axes[0]), r.binned_xy[1], self.m_fBinning)
        return self

    def GetThickness(self, angstrom: bool = False) -> float:
        t = np.float32(self.m_aiSampleEdges[1] - self.m_aiSampleEdges[0])
        return float(t * self.m_fPixSize) if angstrom else float(t)

    def GetLowEdge(self, angstrom: bool = False) -> float:
        return float(np.float32(self.m_aiSampleEdges[0]) * (self.m_fPixSize if angstrom else np.float32(1)))

    def GetHighEdge(self, angstrom: bool = False) -> float:
        return float(np.float32(self.m_aiSampleEdges[1]) * (self.m_fPixSize if angstrom else np.float32(1)))


def recon_series(tilt_series: "TiltSeries", align_param: "AlignParam", vol_z: int, at_bin: float = 1.0,
                 method: int = WBP, local_param: "LocalAlignParam | None" = None, seed=None, start_tilt: int = 0,
                 num_tilts: int | None = None, iterations: int = 0, subsets: int = 1, **plan_kw) -> np.ndarray:
    """The reconstruction step of CAreTomoMain::mRecon / mReconVol
    (AreTomo/CAreTomoMain.cpp:727-761, 809-879) on one GPU: the aligned series
    (CCorrTomoStack with Fourier cropping, rotation by the tilt axes, local
    patches if given), Fourier-binned by at_bin (CBinStack::DoFFT), then WBP or
    SART of thickness vol_z (of the binned series).  The binned series stays on
    the device between the two stages; the volume [by][vol_z][bx & ~1] comes
    back to host memory.  seed: the fill's random table (None: the time, as
    the reference)."""
    import torch
    nx, ny, nt = tilt_series.stk_size
    axes = np.asarray([align_param.GetTiltAxis(i) for i in range(nt)], np.float32)
    st = Stack(nx, ny, nt, shifts=np.asarray([align_param.GetShift(i) for i in range(nt)], np.float32),
               tilt_axes=axes, size_axis=float(axes[0]),
               local_params=None if local_param is None else local_param.params, rand_fill=True, seed=seed,
               bin=at_bin)
    try:
        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.current_stream(dev)
        raw = torch.from_numpy(np.ascontiguousarray(tilt_series.frames, np.float32)).to(dev)
        binned = torch.empty(st.binned_shape, device=dev, dtype=torch.float32)
        st.run_device(raw.data_ptr(), binned.data_ptr(), stream.cuda_stream)
        del raw
    finally:
        st.close()
    kw = dict(plan_kw)
    if method == SART:
        kw.update(start_tilt=start_tilt, num_tilts=nt if num_tilts is None else num_tilts, iterations=iterations,
                  subsets=subsets)
    vol, plan = reconstruct_device(binned, align_param.GetTilts(False)[:nt], vol_z, method=method, stream=stream, **kw)
    try:
        out = vol.cpu().numpy()
    finally:
        plan.close()
    return out


def save_mrc(path: str, frames, pix_size: float = 1.0) -> None:
    """The volume file CAsyncSaveVol::mSaveVol writes (DataUtil/
    CAsyncSaveVol.cpp:82-126): frames [nz][ny][nx] (an array, or a list of
    equal-sized 2-D frames) as a float MRC with the reference writer's header."""
    fr = [np.ascontiguousarray(f, np.float32) for f in frames]
    if not fr or any(f.ndim != 2 or f.shape != fr[0].shape for f in fr):
        raise ValueError("frames must be equal-sized 2-D arrays")
    ny, nx = fr[0].shape
    P = ctypes.c_void_p * len(fr)
    _check(lib().at3r_mrc_write(os.fsencode(path), P(*[f.ctypes.data for f in fr]), nx, ny, len(fr),
                                float(pix_size)))
