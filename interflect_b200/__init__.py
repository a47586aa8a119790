"""interflect_b200: Interflect's surfel-radiosity path on one NVIDIA B200.

Python mirror of the reference crate's stage API over the C ABI in
include/interflect.h (the library is ``lib/libinterflect_b200.so``, built by
``python -m interflect_b200.build``). The stages keep the reference's names
and argument meaning:

    scene = parse(src)                       # scene::parse        (scene.rs:365)
    ctx = Context(device=0); ctx.upload(scene)
    ctx.generate(scene.cfg.surfels)          # surfel::generate    (surfel.rs:147)
    info = ctx.build(cluster_res=8)          # formfactor::build_clusters + build (formfactor.rs:91,153)
    ctx.light_surfels()                      # solve::light_surfels (solve.rs:27)
    stats = ctx.solve(scene.cfg.bounces)     # solve::solve        (solve.rs:47)
    ctx.grid_build()                         # surfel::Grid::build (surfel.rs:71; radius as main.rs:473)
    img = ctx.render_frame(...)              # render_frame + Film::encode (main.rs:229, film.rs:51)

Errors follow the reference: a malformed scene raises ParseError carrying the
diagnostic the reference prints after ``error:``; any device failure raises
DeviceError. There is no CPU fallback: without the compiled library or a CUDA
device every device-side call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# IFX_CHECKED=1 selects the bounds-checked build of the same library (test
# runs only; every scene-array index checked, failures reported as errors).
LIB_PATH = os.path.join(_HERE, "lib", "libinterflect_b200_checked.so" if os.environ.get("IFX_CHECKED") == "1"
                        else "libinterflect_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "interflect")
COMPARE_PATH = os.path.join(_HERE, "bin", "compare")

IFX_OK, IFX_ERR_INVALID, IFX_ERR_PARSE, IFX_ERR_CUDA, IFX_ERR_NOMEM, IFX_ERR_LIMIT, IFX_ERR_TIMEOUT = range(7)
WAIT_LIMIT_DEFAULT = 1 << 22  # IFX_WAIT_LIMIT_DEFAULT
MULTISCENE_WAIT_DEFAULT = 1 << 24  # IFX_MULTISCENE_WAIT_DEFAULT
MODES = {"beauty": 0, "direct": 1, "indirect": 2, "normals": 3, "depth": 4, "steps": 5}

# Every symbol include/interflect.h declares.
EXPORTS = (
    "ifx_scene_parse", "ifx_scene_free", "ifx_scene_get_info", "ifx_scene_set_cfg", "ifx_scene_set_use_bvh",
    "ifx_scene_get_bvh", "ifx_set_wait_limit", "ifx_set_leaf_grid", "ifx_multiscene_set_wait_limit",
    "ifx_ctx_create", "ifx_ctx_destroy", "ifx_last_error", "ifx_get_stats", "ifx_scene_upload",
    "ifx_surfels_generate", "ifx_surfels_upload", "ifx_surfels_count", "ifx_surfels_download",
    "ifx_transfer_build", "ifx_transfer_download", "ifx_clusters_download", "ifx_transfer_row_diag",
    "ifx_transfer_upload", "ifx_light_surfels", "ifx_solve", "ifx_grid_build", "ifx_render_frame",
    "ifx_set_work_counting", "ifx_reset_work", "ifx_get_work", "ifx_timer_start", "ifx_timer_stop",
    "ifx_solve_noalloc", "ifx_surfels_set_emission", "ifx_solve_batched", "ifx_autotune_batched",
    "ifx_surfels_set_albedo", "ifx_lights_set_emission", "ifx_lights_get_emission", "ifx_diff_setup",
    "ifx_diff_forward", "ifx_diff_backward",
    "ifx_multiscene_create", "ifx_multiscene_destroy", "ifx_multiscene_last_error", "ifx_multiscene_add",
    "ifx_multiscene_build", "ifx_multiscene_run", "ifx_multiscene_download", "ifx_set_stage_limit",
    "ifx_clusters_build", "ifx_render_reference", "ifx_frame",
)
NOALLOC_MAX_CLUSTERS = 16384
KERNELS = {"visibility": 0, "closure": 1, "light": 2, "primary": 3, "shadow": 4, "reflect": 5, "shadow2": 6,
           "shade_other": 7, "path": 8}
WORK_COUNTERS = 21


class ParseError(ValueError):
    """A malformed .rad scene (the reference's scene::parse Err)."""


class LimitError(ValueError):
    """A render setting beyond the reference's limits (RenderCfg::validate)."""


class DeviceError(RuntimeError):
    """A CUDA failure, a missing device or a failed device-side check."""


class WaitTimeout(DeviceError):
    """A bounded device-side wait ran out of polls (IFX_ERR_TIMEOUT); the
    call's results are invalid, the context stays usable."""


class _RenderCfg(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("surfels", C.c_uint64), ("bounces", C.c_uint32),
                ("exposure", C.c_float)]


class _Camera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("look", C.c_float * 3), ("up", C.c_float * 3), ("fov", C.c_float)]


class _SceneInfo(C.Structure):
    _fields_ = [("objects", C.c_uint32), ("planes", C.c_uint32), ("lights", C.c_uint32),
                ("sphere_lights", C.c_uint32), ("materials", C.c_uint32), ("bvh_nodes", C.c_uint32),
                ("bounds_lo", C.c_float * 3), ("bounds_hi", C.c_float * 3), ("cfg", _RenderCfg),
                ("camera", _Camera)]


class _TransferInfo(C.Structure):
    _fields_ = [("clusters", C.c_uint64), ("links", C.c_uint64), ("candidates", C.c_uint64), ("evals", C.c_uint64),
                ("interior_rows", C.c_uint64), ("mean_row_sum", C.c_float)]


class _SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("residual", C.c_float)]


class _FrameInfo(C.Structure):
    _fields_ = [("transfer", _TransferInfo), ("light_evals", C.c_uint64), ("solve", _SolveStats),
                ("shade_evals", C.c_uint64), ("ms_frame", C.c_float)]


class _Stats(C.Structure):
    _fields_ = [("kernel_launches", C.c_uint64), ("ms_transfer", C.c_float), ("ms_light", C.c_float),
                ("ms_solve", C.c_float), ("ms_grid", C.c_float), ("ms_shade", C.c_float),
                ("ms_visibility", C.c_float), ("ms_closure", C.c_float), ("ms_primary", C.c_float),
                ("ms_shadow", C.c_float), ("ms_reflect", C.c_float), ("ms_shadow2", C.c_float),
                ("ms_shade_other", C.c_float), ("ms_diff_forward", C.c_float), ("ms_diff_backward", C.c_float)]


class _DiffInfo(C.Structure):
    _fields_ = [("surfels", C.c_uint64), ("lights", C.c_uint64), ("pixels", C.c_uint64),
                ("gather_entries", C.c_uint64), ("links", C.c_uint64), ("bounces", C.c_uint32),
                ("ms_setup", C.c_float)]


_lib_handle = None


def lib() -> C.CDLL:
    """The loaded C-ABI library. Raises DeviceError if it was not built."""
    global _lib_handle
    if _lib_handle is not None:
        return _lib_handle
    if not os.path.exists(LIB_PATH):
        raise DeviceError(f"{LIB_PATH} is missing: run `python -m interflect_b200.build` (CUDA toolkit required)")
    L = C.CDLL(LIB_PATH)
    P, U64, U32, I, F = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_float
    sig = {
        "ifx_scene_parse": (I, [C.c_char_p, C.c_size_t, C.POINTER(P), C.c_char_p, C.c_size_t]),
        "ifx_scene_free": (None, [P]),
        "ifx_scene_get_info": (I, [P, C.POINTER(_SceneInfo)]),
        "ifx_scene_set_cfg": (I, [P, C.POINTER(_RenderCfg), C.c_char_p, C.c_size_t]),
        "ifx_scene_set_use_bvh": (I, [P, I]),
        "ifx_scene_get_bvh": (I, [P, P, P]),
        "ifx_ctx_create": (I, [I, C.POINTER(P)]),
        "ifx_ctx_destroy": (None, [P]),
        "ifx_last_error": (C.c_char_p, [P]),
        "ifx_get_stats": (I, [P, C.POINTER(_Stats)]),
        "ifx_scene_upload": (I, [P, P]),
        "ifx_surfels_generate": (I, [P, U64, C.POINTER(U64)]),
        "ifx_surfels_upload": (I, [P, U64, P, P, P, P]),
        "ifx_surfels_count": (I, [P, C.POINTER(U64)]),
        "ifx_surfels_download": (I, [P, P, P, P, P, P, P, P]),
        "ifx_transfer_build": (I, [P, I, C.POINTER(_TransferInfo)]),
        "ifx_transfer_download": (I, [P, P, P, P]),
        "ifx_clusters_download": (I, [P, P, P, P]),
        "ifx_transfer_row_diag": (I, [P, P, P, P, P]),
        "ifx_transfer_upload": (I, [P, P, U64, P, P]),
        "ifx_light_surfels": (I, [P, C.POINTER(U64)]),
        "ifx_solve": (I, [P, U32, C.POINTER(_SolveStats)]),
        "ifx_grid_build": (I, [P, F]),
        "ifx_render_frame": (I, [P, C.POINTER(_Camera), I, U32, U32, F, P, P, C.POINTER(U64)]),
        "ifx_set_work_counting": (I, [P, I]),
        "ifx_reset_work": (I, [P]),
        "ifx_get_work": (I, [P, I, P, C.POINTER(C.c_double)]),
        "ifx_timer_start": (I, [P]),
        "ifx_timer_stop": (I, [P, C.POINTER(F)]),
        "ifx_solve_noalloc": (I, [I, P, U32, U32, P, P, P, P, P, P, P, P, P, P, P, U32, C.POINTER(_SolveStats),
                                  C.c_char_p, C.c_size_t]),
        "ifx_surfels_set_emission": (I, [P, P]),
        "ifx_solve_batched": (I, [P, U32, P, U32, P, P, P, P]),
        "ifx_autotune_batched": (I, [P, U32, P, C.POINTER(I)]),
        "ifx_surfels_set_albedo": (I, [P, P]),
        "ifx_lights_set_emission": (I, [P, U32, P]),
        "ifx_lights_get_emission": (I, [P, U32, P]),
        "ifx_diff_setup": (I, [P, C.POINTER(_Camera), U32, U32, U32, C.POINTER(_DiffInfo)]),
        "ifx_diff_forward": (I, [P, P, P, P]),
        "ifx_diff_backward": (I, [P, P, P, P]),
        "ifx_multiscene_create": (I, [I, C.POINTER(P)]),
        "ifx_multiscene_destroy": (None, [P]),
        "ifx_multiscene_last_error": (C.c_char_p, [P]),
        "ifx_multiscene_add": (I, [P, P, C.POINTER(_Camera), U32, U32, U32, C.POINTER(I)]),
        "ifx_multiscene_build": (I, [P, I, C.POINTER(I), C.POINTER(I)]),
        "ifx_multiscene_run": (I, [P, C.POINTER(F)]),
        "ifx_multiscene_download": (I, [P, I, P, P, C.POINTER(_SolveStats)]),
        "ifx_set_stage_limit": (I, [P, U32]),
        "ifx_set_wait_limit": (I, [P, U32]),
        "ifx_set_leaf_grid": (I, [P, I]),
        "ifx_multiscene_set_wait_limit": (I, [P, U32]),
        "ifx_clusters_build": (I, [P, I, C.POINTER(U64)]),
        "ifx_render_reference": (I, [P, C.POINTER(_Camera), U32, U32, U32, F, P, P]),
        "ifx_frame": (I, [P, I, U32, C.POINTER(_Camera), I, U32, U32, F, P, P, C.POINTER(_FrameInfo)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib_handle = L
    return L


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class RenderCfg:
    width: int
    height: int
    surfels: int
    bounces: int
    exposure: float


@dataclass
class SceneInfo:
    objects: int
    planes: int
    lights: int
    sphere_lights: int
    materials: int
    bvh_nodes: int
    bounds_lo: tuple
    bounds_hi: tuple
    cfg: RenderCfg
    camera: dict


@dataclass
class TransferInfo:
    clusters: int
    links: int
    candidates: int
    evals: int
    interior_rows: int
    mean_row_sum: float


@dataclass
class SolveStats:
    iterations: int
    residual: float


class Scene:
    """A parsed .rad scene (host side): scene::parse plus Bvh::build."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ifx_scene_free(self._h)
            self._h = None

    @property
    def info(self) -> SceneInfo:
        i = _SceneInfo()
        lib().ifx_scene_get_info(self._h, C.byref(i))
        c = i.cfg
        cam = i.camera
        return SceneInfo(i.objects, i.planes, i.lights, i.sphere_lights, i.materials, i.bvh_nodes,
                         tuple(i.bounds_lo), tuple(i.bounds_hi),
                         RenderCfg(c.width, c.height, c.surfels, c.bounces, c.exposure),
                         dict(pos=tuple(cam.pos), look=tuple(cam.look), up=tuple(cam.up), fov=cam.fov))

    @property
    def cfg(self) -> RenderCfg:
        return self.info.cfg

    @property
    def diag(self) -> float:
        i = self.info
        lo = np.array(i.bounds_lo, np.float32)
        hi = np.array(i.bounds_hi, np.float32)
        d = hi - lo
        return float(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))

    def set_cfg(self, width=None, height=None, surfels=None, bounces=None, exposure=None) -> None:
        """CLI overrides, re-validated (main.rs:394-413). Raises LimitError."""
        c = self.cfg
        rc = _RenderCfg(width if width is not None else c.width, height if height is not None else c.height,
                        surfels if surfels is not None else c.surfels, bounces if bounces is not None else c.bounces,
                        exposure if exposure is not None else c.exposure)
        err = C.create_string_buffer(512)
        r = lib().ifx_scene_set_cfg(self._h, C.byref(rc), err, 512)
        if r != IFX_OK:
            raise LimitError(err.value.decode())

    def bvh(self):
        """(nodes as 9 u32 words each, leaf object order), see ifx_scene_get_bvh."""
        i = self.info
        nodes = np.zeros((i.bvh_nodes, 9), np.uint32)
        order = np.zeros(i.objects, np.uint32)
        lib().ifx_scene_get_bvh(self._h, _ptr(nodes), _ptr(order))
        return nodes, order

    def set_use_bvh(self, on: bool) -> None:
        lib().ifx_scene_set_use_bvh(self._h, 1 if on else 0)


def parse(src: str) -> Scene:
    """scene::parse (scene.rs:365-571). Raises ParseError on malformed input."""
    b = src.encode()
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    r = lib().ifx_scene_parse(b, len(b), C.byref(h), err, 512)
    if r != IFX_OK:
        raise ParseError(err.value.decode())
    return Scene(h)


def load(path: str) -> Scene:
    with open(path) as f:
        return parse(f.read())


def _out(buf, shape, dtype, want: bool):
    """The caller's output array (checked: C-contiguous, shape, dtype), a new
    one, or None."""
    if buf is not None:
        if buf.shape != shape or buf.dtype != dtype or not buf.flags["C_CONTIGUOUS"] or not buf.flags["WRITEABLE"]:
            raise ValueError(f"output array must be a writeable C-contiguous {np.dtype(dtype).name} array of "
                             f"shape {shape}")
        return buf
    return np.zeros(shape, dtype) if want else None


def camera(pos, look, up=(0.0, 1.0, 0.0), fov=40.0) -> _Camera:
    c = _Camera()
    c.pos[:] = pos
    c.look[:] = look
    c.up[:] = up
    c.fov = fov
    return c


class Context:
    """One GPU, one CUDA stream, the device state of one scene's pipeline."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        r = lib().ifx_ctx_create(device, C.byref(h))
        if r != IFX_OK:
            raise DeviceError(f"ifx_ctx_create(device={device}) failed with status {r} (no usable CUDA device?)")
        self._h = h
        self.scene: Scene | None = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ifx_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, r: int, what: str) -> None:
        if r != IFX_OK:
            msg = lib().ifx_last_error(self._h).decode(errors="replace")
            if r == IFX_ERR_LIMIT:
                raise LimitError(f"{what}: {msg}")
            if r == IFX_ERR_TIMEOUT:
                raise WaitTimeout(f"{what} failed ({r}): {msg}")
            raise DeviceError(f"{what} failed ({r}): {msg}")

    # -- scene / surfels ------------------------------------------------
    def upload(self, scene: Scene) -> None:
        self._check(lib().ifx_scene_upload(self._h, scene._h), "scene upload")
        self.scene = scene

    def generate(self, target: int) -> int:
        """surfel::generate: returns the placed surfel count."""
        n = C.c_uint64()
        self._check(lib().ifx_surfels_generate(self._h, target, C.byref(n)), "surfel generation")
        return n.value

    def upload_surfels(self, p, n, albedo, area) -> None:
        p, n, albedo = (np.ascontiguousarray(x, np.float32).reshape(-1, 3) for x in (p, n, albedo))
        area = np.ascontiguousarray(area, np.float32).reshape(-1)
        self._check(lib().ifx_surfels_upload(self._h, len(area), _ptr(p), _ptr(n), _ptr(albedo), _ptr(area)),
                    "surfel upload")

    @property
    def n_surfels(self) -> int:
        v = C.c_uint64()
        lib().ifx_surfels_count(self._h, C.byref(v))
        return v.value

    def surfels(self) -> dict:
        k = self.n_surfels
        out = {f: np.zeros((k, 3), np.float32) for f in ("p", "n", "albedo", "direct", "irr", "rad")}
        out["area"] = np.zeros(k, np.float32)
        self._check(lib().ifx_surfels_download(self._h, *(_ptr(out[f]) for f in
                                                          ("p", "n", "albedo", "area", "direct", "irr", "rad"))),
                    "surfel download")
        return out

    # -- transfer ---------------------------------------------------------
    def build(self, cluster_res: int = 8) -> TransferInfo:
        """formfactor::build_clusters followed by formfactor::build."""
        i = _TransferInfo()
        self._check(lib().ifx_transfer_build(self._h, cluster_res, C.byref(i)), "transfer build")
        self._tinfo = TransferInfo(i.clusters, i.links, i.candidates, i.evals, i.interior_rows, i.mean_row_sum)
        return self._tinfo

    def build_clusters(self, cluster_res: int = 8) -> int:
        """formfactor::build_clusters alone; returns the cluster count."""
        nc = C.c_uint64()
        self._check(lib().ifx_clusters_build(self._h, cluster_res, C.byref(nc)), "cluster build")
        return nc.value

    def transfer(self) -> dict:
        k = self.n_surfels
        starts = np.zeros(k + 1, np.uint32)
        self._check(lib().ifx_transfer_download(self._h, _ptr(starts), None, None), "transfer download")
        links = int(starts[-1])
        idx = np.zeros(links, np.uint32)
        w = np.zeros(links, np.float32)
        self._check(lib().ifx_transfer_download(self._h, None, _ptr(idx), _ptr(w)), "transfer download")
        return dict(starts=starts, idx=idx, w=w)

    def clusters(self, nc: int) -> dict:
        pnar = np.zeros((nc, 8), np.float32)
        off = np.zeros(nc + 1, np.uint32)
        mem = np.zeros(self.n_surfels, np.uint32)
        self._check(lib().ifx_clusters_download(self._h, _ptr(pnar), _ptr(off), _ptr(mem)), "cluster download")
        return dict(p=pnar[:, 0:3], n=pnar[:, 3:6], area=pnar[:, 6], radius=pnar[:, 7], offsets=off, members=mem)

    def row_diag(self) -> dict:
        k = self.n_surfels
        out = dict(row_sum=np.zeros(k, np.float32), row_sky=np.zeros(k, np.float32),
                   row_evals=np.zeros(k, np.uint64), cand_count=np.zeros(k, np.uint32))
        self._check(lib().ifx_transfer_row_diag(self._h, _ptr(out["row_sum"]), _ptr(out["row_sky"]),
                                                _ptr(out["row_evals"]), _ptr(out["cand_count"])), "row diag")
        return out

    def upload_transfer(self, starts, idx, w) -> None:
        starts = np.ascontiguousarray(starts, np.uint32)
        idx = np.ascontiguousarray(idx, np.uint32)
        w = np.ascontiguousarray(w, np.float32)
        self._check(lib().ifx_transfer_upload(self._h, _ptr(starts), len(idx), _ptr(idx), _ptr(w)),
                    "transfer upload")

    # -- solve --------------------------------------------------------------
    def light_surfels(self) -> int:
        """solve::light_surfels: returns its SDF evaluation count."""
        e = C.c_uint64()
        self._check(lib().ifx_light_surfels(self._h, C.byref(e)), "light_surfels")
        return e.value

    def solve(self, max_bounces: int) -> SolveStats:
        s = _SolveStats()
        self._check(lib().ifx_solve(self._h, max_bounces, C.byref(s)), "solve")
        return SolveStats(s.iterations, s.residual)

    # -- relighting -----------------------------------------------------------
    def set_emission(self, E) -> None:
        """direct = rad = E, irr = 0: the solve's source for one relighting."""
        E = np.ascontiguousarray(E, np.float32).reshape(-1, 3)
        self._check(lib().ifx_surfels_set_emission(self._h, _ptr(E)), "set_emission")

    def solve_batched(self, E, max_bounces: int, outputs: bool = True, R: int | None = None):
        """R relighting right-hand sides E (R x n x 3) as one SpMM solve; E
        None reuses the previous call's right-hand sides (resident on the
        device; pass R). Returns (rad R x n x 3, irr R x n x 3, iterations[R],
        residual[R]); rad and irr are None when outputs is False."""
        if E is not None:
            E = np.ascontiguousarray(E, np.float32)
            R = E.shape[0]
        shape = (R, self.n_surfels, 3)
        rad = np.zeros(shape, np.float32) if outputs else None
        irr = np.zeros(shape, np.float32) if outputs else None
        it = np.zeros(R, np.uint32)
        res = np.zeros(R, np.float32)
        self._check(lib().ifx_solve_batched(self._h, R, _ptr(E), max_bounces, _ptr(rad), _ptr(irr), _ptr(it),
                                            _ptr(res)), "solve_batched")
        return rad, irr, it, res

    def autotune_batched(self, E) -> int:
        E = np.ascontiguousarray(E, np.float32)
        best = C.c_int()
        self._check(lib().ifx_autotune_batched(self._h, E.shape[0], _ptr(E), C.byref(best)), "autotune_batched")
        return best.value

    # -- shade --------------------------------------------------------------
    def grid_build(self, radius: float = 0.0) -> None:
        self._check(lib().ifx_grid_build(self._h, radius), "grid build")

    def render_frame(self, width: int, height: int, mode="beauty", cam=None, exposure: float | None = None,
                     linear: bool = True, srgb: bool = True, out_linear=None, out_srgb=None):
        """render_frame + Film::encode. Returns (linear f32 HxWx3 | None, u8 HxWx3 | None, evals)."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        if exposure is None:
            exposure = self.scene.cfg.exposure if self.scene is not None else 1.0
        lin = _out(out_linear, (height, width, 3), np.float32, linear)
        s8 = _out(out_srgb, (height, width, 3), np.uint8, srgb)
        e = C.c_uint64()
        self._check(lib().ifx_render_frame(self._h, C.byref(cam) if cam is not None else None, m, width, height,
                                           exposure, _ptr(lin), _ptr(s8), C.byref(e)), "render_frame")
        return lin, s8, e.value

    def frame(self, width: int, height: int, mode="beauty", cluster_res: int = 8, max_bounces: int | None = None,
              cam=None, exposure: float | None = None, linear: bool = True, srgb: bool = True, out_linear=None,
              out_srgb=None) -> dict:
        """The transfer build, light_surfels, solve, grid and render_frame in
        one call, the GI-independent shading passes overlapped with the GI
        stages. Returns dict(linear, srgb, transfer, light_evals, solve,
        shade_evals, ms_frame). `out_linear` / `out_srgb` (optional) are
        arrays to fill instead of new ones, e.g. reused across frames."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        cfg = self.scene.cfg if self.scene is not None else None
        if exposure is None:
            exposure = cfg.exposure if cfg is not None else 1.0
        if max_bounces is None:
            max_bounces = cfg.bounces if cfg is not None else 16
        lin = _out(out_linear, (height, width, 3), np.float32, linear)
        s8 = _out(out_srgb, (height, width, 3), np.uint8, srgb)
        fi = _FrameInfo()
        self._check(lib().ifx_frame(self._h, cluster_res, max_bounces, C.byref(cam) if cam is not None else None, m,
                                    width, height, exposure, _ptr(lin), _ptr(s8), C.byref(fi)), "frame")
        t = fi.transfer
        if m in (MODES["beauty"], MODES["indirect"]):
            self._tinfo = TransferInfo(t.clusters, t.links, t.candidates, t.evals, t.interior_rows, t.mean_row_sum)
        return dict(linear=lin, srgb=s8,
                    transfer=TransferInfo(t.clusters, t.links, t.candidates, t.evals, t.interior_rows,
                                          t.mean_row_sum),
                    light_evals=fi.light_evals, solve=SolveStats(fi.solve.iterations, fi.solve.residual),
                    shade_evals=fi.shade_evals, ms_frame=fi.ms_frame)

    def render_reference(self, width: int, height: int, spp: int = 512, cam=None, exposure: float | None = None,
                         linear: bool = True, srgb: bool = True, out_linear=None, out_srgb=None):
        """--mode reference: the path tracer of reference.rs. Returns (linear | None, u8 | None)."""
        if exposure is None:
            exposure = self.scene.cfg.exposure if self.scene is not None else 1.0
        lin = _out(out_linear, (height, width, 3), np.float32, linear)
        s8 = _out(out_srgb, (height, width, 3), np.uint8, srgb)
        self._check(lib().ifx_render_reference(self._h, C.byref(cam) if cam is not None else None, width, height, spp,
                                               exposure, _ptr(lin), _ptr(s8)), "render_reference")
        return lin, s8

    def stats(self) -> dict:
        s = _Stats()
        lib().ifx_get_stats(self._h, C.byref(s))
        return {f: getattr(s, f) for f, _ in _Stats._fields_}

    # -- differentiation ----------------------------------------------------
    @property
    def n_lights(self) -> int:
        i = self.scene.info if self.scene is not None else None
        return 0 if i is None else i.lights + i.sphere_lights

    def set_albedo(self, rho) -> None:
        """Per-surfel albedo override (n x 3)."""
        rho = np.ascontiguousarray(rho, np.float32).reshape(-1, 3)
        if len(rho) != self.n_surfels:
            raise ValueError(f"albedo has {len(rho)} rows for {self.n_surfels} surfels")
        self._check(lib().ifx_surfels_set_albedo(self._h, _ptr(rho)), "set_albedo")

    def set_light_emission(self, emit) -> None:
        """Per-light emission (nl x 3: quad lights, then sphere lights)."""
        emit = np.ascontiguousarray(emit, np.float32).reshape(-1, 3)
        self._check(lib().ifx_lights_set_emission(self._h, len(emit), _ptr(emit)), "set_light_emission")

    def light_emission(self) -> np.ndarray:
        out = np.zeros((self.n_lights, 3), np.float32)
        self._check(lib().ifx_lights_get_emission(self._h, len(out), _ptr(out)), "light_emission")
        return out

    def diff_setup(self, width: int, height: int, bounces: int, cam=None) -> dict:
        """Prepares the differentiable beauty frame (fixed bounce count)."""
        i = _DiffInfo()
        self._check(lib().ifx_diff_setup(self._h, C.byref(cam) if cam is not None else None, width, height,
                                         bounces, C.byref(i)), "diff_setup")
        self._diff_shape = (height, width)
        return {f: getattr(i, f) for f, _ in _DiffInfo._fields_}

    def diff_forward(self, rho=None, emit=None) -> np.ndarray:
        """The prepared frame (H x W x 3 linear f32) for albedo rho and emission emit."""
        if rho is not None:
            rho = np.ascontiguousarray(rho, np.float32).reshape(-1, 3)
            if len(rho) != self.n_surfels:
                raise ValueError(f"albedo has {len(rho)} rows for {self.n_surfels} surfels")
        if emit is not None:
            emit = np.ascontiguousarray(emit, np.float32).reshape(-1, 3)
            if len(emit) != self.n_lights:
                raise ValueError(f"emission has {len(emit)} rows for {self.n_lights} lights")
        img = np.zeros(self._diff_shape + (3,), np.float32)
        self._check(lib().ifx_diff_forward(self._h, _ptr(rho), _ptr(emit), _ptr(img)), "diff_forward")
        return img

    def diff_backward(self, grad_image) -> tuple[np.ndarray, np.ndarray]:
        """(dL/drho n x 3, dL/demit nl x 3) for dL/dimage of the last diff_forward."""
        g = np.ascontiguousarray(grad_image, np.float32).reshape(self._diff_shape + (3,))
        gr = np.zeros((self.n_surfels, 3), np.float32)
        ge = np.zeros((self.n_lights, 3), np.float32)
        self._check(lib().ifx_diff_backward(self._h, _ptr(g), _ptr(gr), _ptr(ge)), "diff_backward")
        return gr, ge

    # -- measurement ----------------------------------------------------------
    def set_work_counting(self, on: bool) -> None:
        """Instrumented kernels (for work/FLOP accounting only, never for timing)."""
        self._check(lib().ifx_set_work_counting(self._h, 1 if on else 0), "set_work_counting")

    def reset_work(self) -> None:
        self._check(lib().ifx_reset_work(self._h), "reset_work")

    def work(self, kernel: str) -> tuple[np.ndarray, float]:
        counts = np.zeros(WORK_COUNTERS, np.uint64)
        fl = C.c_double()
        self._check(lib().ifx_get_work(self._h, KERNELS[kernel], _ptr(counts), C.byref(fl)), "get_work")
        return counts, fl.value

    def set_wait_limit(self, polls: int | None) -> None:
        """Poll budget of the bounded device-side waits (None: the default);
        0 makes every wait give up at once, for tests of that error path."""
        self._check(lib().ifx_set_wait_limit(self._h, WAIT_LIMIT_DEFAULT if polls is None else polls),
                    "set_wait_limit")

    def set_leaf_grid(self, on: bool) -> None:
        """Whether the next upload builds the per-cell leaf lists of large
        BVHs for cone-shadow marches (results are identical either way)."""
        self._check(lib().ifx_set_leaf_grid(self._h, 1 if on else 0), "set_leaf_grid")

    def set_stage_limit(self, max_bytes: int) -> None:
        """Largest geometry program staged in shared memory per CTA (tuning only)."""
        self._check(lib().ifx_set_stage_limit(self._h, max_bytes), "set_stage_limit")

    def timer_start(self) -> None:
        self._check(lib().ifx_timer_start(self._h), "timer_start")

    def timer_stop(self) -> float:
        ms = C.c_float()
        self._check(lib().ifx_timer_stop(self._h, C.byref(ms)), "timer_stop")
        return ms.value


def solve_noalloc(device: int, stream: int, n: int, nc: int, p_area4: int, direct4: int, albedo4: int, irr4: int,
                  rad4: int, cluster_p_area4: int, cluster_ranges: int, members: int, starts: int, idx: int, w: int,
                  max_bounces: int) -> SolveStats:
    """The Jacobi solve on caller-owned device buffers (integer device
    addresses) with no allocation by the library, for callers that cannot
    let it allocate GPU memory (see ifx_solve_noalloc in interflect.h for the
    layouts and the IFX_NOALLOC_MAX_CLUSTERS limit). Raises LimitError above
    that limit and DeviceError on CUDA failures."""
    st = _SolveStats()
    err = C.create_string_buffer(256)
    r = lib().ifx_solve_noalloc(device, stream or None, n, nc, p_area4, direct4, albedo4, irr4, rad4,
                                cluster_p_area4, cluster_ranges, members, starts, idx, w, max_bounces,
                                C.byref(st), err, 256)
    if r == IFX_ERR_LIMIT:
        raise LimitError(err.value.decode())
    if r != IFX_OK:
        raise DeviceError(f"ifx_solve_noalloc failed ({r}): {err.value.decode()}")
    return SolveStats(st.iterations, st.residual)


class MultiScene:
    """Many scenes' solve + shade in one persistent launch replayed from a
    CUDA graph (ifx_multiscene_* in interflect.h). Member contexts must stay
    alive, and unused for other rendering, while they belong to it."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        r = lib().ifx_multiscene_create(device, C.byref(h))
        if r != IFX_OK:
            raise DeviceError(f"ifx_multiscene_create(device={device}) failed with status {r}")
        self._h = h
        self._members: list[tuple[Context, int, int]] = []

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ifx_multiscene_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, r: int, what: str) -> None:
        if r != IFX_OK:
            msg = lib().ifx_multiscene_last_error(self._h).decode(errors="replace")
            if r == IFX_ERR_LIMIT:
                raise LimitError(f"{what}: {msg}")
            if r == IFX_ERR_TIMEOUT:
                raise WaitTimeout(f"{what} failed ({r}): {msg}")
            raise DeviceError(f"{what} failed ({r}): {msg}")

    def add(self, ctx: Context, width: int, height: int, max_bounces: int, cam=None) -> int:
        i = C.c_int()
        self._check(lib().ifx_multiscene_add(self._h, ctx._h, C.byref(cam) if cam is not None else None, width,
                                             height, max_bounces, C.byref(i)), "multiscene add")
        self._members.append((ctx, width, height))
        return i.value

    def set_wait_limit(self, polls: int | None) -> None:
        """Poll budget of the packed launch's grid barriers from the next
        build (None: the default); 0 makes each barrier give up at once."""
        self._check(lib().ifx_multiscene_set_wait_limit(self._h, MULTISCENE_WAIT_DEFAULT if polls is None else polls),
                    "set_wait_limit")

    def build(self, autotune: bool = True) -> tuple[int, int]:
        g, b = C.c_int(), C.c_int()
        self._check(lib().ifx_multiscene_build(self._h, 1 if autotune else 0, C.byref(g), C.byref(b)),
                    "multiscene build")
        return g.value, b.value

    def run(self) -> float:
        ms = C.c_float()
        self._check(lib().ifx_multiscene_run(self._h, C.byref(ms)), "multiscene run")
        return ms.value

    def download(self, index: int, linear: bool = True, srgb: bool = True):
        """(linear H x W x 3 | None, u8 H x W x 3 | None, SolveStats) of scene `index`."""
        _, w, h = self._members[index]
        lin = np.zeros((h, w, 3), np.float32) if linear else None
        s8 = np.zeros((h, w, 3), np.uint8) if srgb else None
        st = _SolveStats()
        self._check(lib().ifx_multiscene_download(self._h, index, _ptr(lin), _ptr(s8), C.byref(st)),
                    "multiscene download")
        return lin, s8, SolveStats(st.iterations, st.residual)


def cuda_available() -> bool:
    """True when a CUDA device is visible to the CUDA runtime."""
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
