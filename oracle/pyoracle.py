"""Oracle (test infrastructure only): ctypes bindings to the CPU restatement
of the reference path (oracle/_build/liboracle.so, built by `make -C oracle`).

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module; it is the checker, never part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
RENDER_BIN = os.path.join(HERE, "_build", "oracle_render")

MODES = {"beauty": 0, "direct": 1, "indirect": 2, "normals": 3, "depth": 4, "steps": 5, "reference": 6}

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, I, I64, F, U32 = C.c_void_p, C.c_int, C.c_int64, C.c_float, C.c_uint32
        sig = {
            "orc_create": (P, []), "orc_destroy": (None, [P]), "orc_error": (C.c_char_p, [P]),
            "orc_set_threads": (None, [P, I]), "orc_set_use_bvh": (None, [P, I]),
            "orc_parse": (I, [P, C.c_char_p]), "orc_scene_info": (I, [P, P, P, P]),
            "orc_bvh": (I, [P, P, P]), "orc_dist_mat": (I, [P, I64, P, P, P]), "orc_normal": (I, [P, I64, P, P]),
            "orc_soft_shadow": (I, [P, I64, P, P, P, P, P, P, P]),
            "orc_trace": (I, [P, I64, P, P, F, F, P, P, P, P, P]),
            "orc_quad_form_factor": (F, [P]), "orc_form_factor_at": (F, [P, P, P]),
            "orc_srgb": (C.c_uint8, [F]), "orc_aces": (None, [P, P]),
            "orc_generate": (I64, [P, I64]), "orc_set_surfels": (I, [P, I64, P, P, P, P]),
            "orc_surfel_count": (I64, [P]), "orc_get_surfels": (I, [P, P, P, P, P, P, P, P]),
            "orc_set_surfel_state": (I, [P, P, P, P]),
            "orc_build_clusters": (I64, [P, I]), "orc_get_clusters": (I, [P, P, P, P]),
            "orc_build_transfer": (I, [P, P, P]), "orc_build_transfer_sampled": (I, [P, I64, P, P]),
            "orc_light_surfels_sampled": (I64, [P, I64]), "orc_get_transfer": (I, [P, P, P, P, P, P, P, P]),
            "orc_set_transfer": (I, [P, I64, P, I64, P, P]),
            "orc_light_surfels": (I64, [P]), "orc_solve": (I, [P, U32, P, P]),
            "orc_build_grid": (I, [P, P, P]), "orc_get_grid": (I, [P, P, P]), "orc_gather": (I, [P, I64, P, P, P]),
            "orc_camera": (I, [P, P, P, F, U32, U32, P]),
            "orc_render": (I64, [P, I, U32, U32, P, P, U32, U32]), "orc_get_film": (I, [P, P]),
            "orc_encode": (I, [P, F, I, P]), "orc_counters": (None, [I, I, P]),
            "orc_solve_ex": (I, [P, U32, I, P, P]), "orc_set_spp": (None, [P, U32]), "orc_set_emission": (I, [P, I64, P]),
            "orc_get_emission": (I, [P, P]), "orc_diff_build": (I, [P, U32, U32, P]),
            "orc_diff_loss": (C.c_double, [P, P, P, I, P, P]), "orc_diff_grad": (C.c_double, [P, P, P, I, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def f32(a):
    return np.ascontiguousarray(a, np.float32)


class OracleError(ValueError):
    pass


class Oracle:
    """One scene and its pipeline state in the CPU restatement."""

    def __init__(self, src: str | None = None, threads: int = 1):
        self.h = lib().orc_create()
        lib().orc_set_threads(self.h, threads)
        if src is not None:
            self.parse(src)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_threads(self, n: int) -> None:
        lib().orc_set_threads(self.h, n)

    def set_use_bvh(self, on: bool) -> None:
        lib().orc_set_use_bvh(self.h, 1 if on else 0)

    def parse(self, src: str) -> None:
        if lib().orc_parse(self.h, src.encode()) != 0:
            raise OracleError(lib().orc_error(self.h).decode())

    def info(self) -> dict:
        out = np.zeros(10, np.int64)
        b = np.zeros(6, np.float32)
        e = np.zeros(1, np.float32)
        lib().orc_scene_info(self.h, _p(out), _p(b), _p(e))
        keys = ["objects", "planes", "lights", "materials", "bvh_nodes", "width", "height", "surfels", "bounces",
                "sphere_lights"]
        d = {k: int(v) for k, v in zip(keys, out)}
        d["lo"], d["hi"], d["exposure"] = b[:3].copy(), b[3:].copy(), float(e[0])
        return d

    def bvh(self):
        n = self.info()["bvh_nodes"]
        nodes = np.zeros((n, 9), np.float32)
        order = np.zeros(self.info()["objects"], np.uint32)
        lib().orc_bvh(self.h, _p(nodes), _p(order))
        return nodes, order

    def dist_mat(self, pts):
        pts = f32(pts).reshape(-1, 3)
        d = np.zeros(len(pts), np.float32)
        m = np.zeros(len(pts), np.uint32)
        lib().orc_dist_mat(self.h, len(pts), _p(pts), _p(d), _p(m))
        return d, m

    def normal(self, pts):
        pts = f32(pts).reshape(-1, 3)
        out = np.zeros_like(pts)
        lib().orc_normal(self.h, len(pts), _p(pts), _p(out))
        return out

    def soft_shadow(self, ro, rd, tmin, tmax, k):
        ro, rd = f32(ro).reshape(-1, 3), f32(rd).reshape(-1, 3)
        n = len(ro)
        tmin, tmax, k = (np.broadcast_to(f32(x), (n,)).copy() for x in (tmin, tmax, k))
        vis = np.zeros(n, np.float32)
        steps = np.zeros(n, np.uint32)
        lib().orc_soft_shadow(self.h, n, _p(ro), _p(rd), _p(tmin), _p(tmax), _p(k), _p(vis), _p(steps))
        return vis, steps

    def generate(self, target: int) -> int:
        return int(lib().orc_generate(self.h, target))

    def set_surfels(self, p, n, albedo, area) -> None:
        p, n, albedo = (f32(x).reshape(-1, 3) for x in (p, n, albedo))
        area = f32(area).reshape(-1)
        lib().orc_set_surfels(self.h, len(area), _p(p), _p(n), _p(albedo), _p(area))

    def surfels(self) -> dict:
        k = int(lib().orc_surfel_count(self.h))
        out = {f: np.zeros((k, 3), np.float32) for f in ("p", "n", "albedo", "direct", "irr", "rad")}
        out["area"] = np.zeros(k, np.float32)
        lib().orc_get_surfels(self.h, *(_p(out[f]) for f in ("p", "n", "albedo", "area", "direct", "irr", "rad")))
        return out

    def set_surfel_state(self, direct=None, irr=None, rad=None) -> None:
        lib().orc_set_surfel_state(self.h, _p(None if direct is None else f32(direct)),
                                   _p(None if irr is None else f32(irr)), _p(None if rad is None else f32(rad)))

    def build_clusters(self, res: int = 8) -> int:
        r = int(lib().orc_build_clusters(self.h, res))
        if r < 0:
            raise OracleError(lib().orc_error(self.h).decode())
        return r

    def clusters(self, nc: int, n: int) -> dict:
        pnar = np.zeros((nc, 8), np.float32)
        off = np.zeros(nc + 1, np.uint32)
        mem = np.zeros(n, np.uint32)
        lib().orc_get_clusters(self.h, _p(pnar), _p(off), _p(mem))
        return dict(p=pnar[:, 0:3], n=pnar[:, 3:6], area=pnar[:, 6], radius=pnar[:, 7], offsets=off, members=mem)

    def build_transfer(self, stride: int = 1) -> dict:
        """stride > 1: only rows i % stride == 0 are built (a timing sample);
        the other rows stay empty."""
        info = np.zeros(4, np.int64)
        mean = np.zeros(1, np.float32)
        lib().orc_build_transfer_sampled(self.h, stride, _p(info), _p(mean))
        return dict(clusters=int(info[0]), links=int(info[1]), evals=int(info[2]), interior_rows=int(info[3]),
                    mean_row_sum=float(mean[0]))

    def transfer(self, n: int, links: int) -> dict:
        t = dict(starts=np.zeros(n + 1, np.uint32), idx=np.zeros(links, np.uint32), w=np.zeros(links, np.float32),
                 row_sum=np.zeros(n, np.float32), row_sky=np.zeros(n, np.float32),
                 row_evals=np.zeros(n, np.uint64), cand_count=np.zeros(n, np.uint32))
        lib().orc_get_transfer(self.h, *(_p(t[k]) for k in ("starts", "idx", "w", "row_sum", "row_sky", "row_evals",
                                                          "cand_count")))
        return t

    def set_transfer(self, starts, idx, w) -> None:
        starts = np.ascontiguousarray(starts, np.uint32)
        idx = np.ascontiguousarray(idx, np.uint32)
        w = f32(w)
        lib().orc_set_transfer(self.h, len(starts) - 1, _p(starts), len(idx), _p(idx), _p(w))

    def light_surfels(self, stride: int = 1) -> int:
        """stride > 1: only surfels i % stride == 0 are lit (a timing sample)."""
        return int(lib().orc_light_surfels_sampled(self.h, stride))

    def solve(self, max_bounces: int, fixed: bool = False):
        """fixed: exactly max_bounces bounces (no residual exit)."""
        it = np.zeros(1, np.uint32)
        res = np.zeros(1, np.float32)
        if lib().orc_solve_ex(self.h, max_bounces, 1 if fixed else 0, _p(it), _p(res)) != 0:
            raise OracleError(lib().orc_error(self.h).decode())
        return int(it[0]), float(res[0])

    def set_emission(self, e) -> None:
        """Per-light emission (quad lights, then sphere lights), nl x 3."""
        e = f32(e).reshape(-1, 3)
        if lib().orc_set_emission(self.h, len(e), _p(e)) != 0:
            raise OracleError("emission count does not match the scene's lights")

    def emission(self):
        i = self.info()
        out = np.zeros((i["lights"] + i["sphere_lights"], 3), np.float32)
        lib().orc_get_emission(self.h, _p(out))
        return out

    def diff_build(self, width: int, height: int) -> tuple[int, int, int]:
        """FP64 differentiable model of the scene camera; (surfels, lights, pixels)."""
        d = np.zeros(3, np.int64)
        if lib().orc_diff_build(self.h, width, height, _p(d)) != 0:
            raise OracleError(lib().orc_error(self.h).decode())
        self._diff_dims = tuple(int(v) for v in d)
        return self._diff_dims

    def diff_loss(self, rho, e, K: int, target=None):
        """(L, image P x 3) of the FP64 model; L = sum (image - target)^2."""
        N, nl, P = self._diff_dims
        rho = np.ascontiguousarray(rho, np.float64).reshape(N, 3)
        e = np.ascontiguousarray(e, np.float64).reshape(nl, 3)
        t = None if target is None else np.ascontiguousarray(target, np.float64).reshape(P, 3)
        img = np.zeros((P, 3), np.float64)
        L = lib().orc_diff_loss(self.h, _p(rho), _p(e), K, _p(t), _p(img))
        return float(L), img

    def diff_grad(self, rho, e, K: int, target=None):
        """(L, dL/drho N x 3, dL/de nl x 3) of the FP64 model."""
        N, nl, P = self._diff_dims
        rho = np.ascontiguousarray(rho, np.float64).reshape(N, 3)
        e = np.ascontiguousarray(e, np.float64).reshape(nl, 3)
        t = None if target is None else np.ascontiguousarray(target, np.float64).reshape(P, 3)
        gr = np.zeros((N, 3), np.float64)
        ge = np.zeros((nl, 3), np.float64)
        L = lib().orc_diff_grad(self.h, _p(rho), _p(e), K, _p(t), _p(gr), _p(ge))
        return float(L), gr, ge

    def build_grid(self):
        r = np.zeros(1, np.float32)
        dims = np.zeros(3, np.int32)
        lib().orc_build_grid(self.h, _p(r), _p(dims))
        return float(r[0]), dims

    def grid(self, n: int, ncells: int):
        starts = np.zeros(ncells + 1, np.uint32)
        items = np.zeros(n, np.uint32)
        lib().orc_get_grid(self.h, _p(starts), _p(items))
        return starts, items

    def gather(self, p, n):
        p, n = f32(p).reshape(-1, 3), f32(n).reshape(-1, 3)
        out = np.zeros_like(p)
        lib().orc_gather(self.h, len(p), _p(p), _p(n), _p(out))
        return out

    def render(self, width: int, height: int, mode="beauty", pos=None, look=None, rows=None, spp: int = 512):
        """Linear film (H x W x 3) and the SDF evaluation count. `rows` = (y0, y1) shades only those rows;
        `spp` is the path tracer's samples per pixel (mode "reference")."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        lib().orc_set_spp(self.h, spp)
        y0, y1 = rows if rows else (0, 0)
        ev = lib().orc_render(self.h, m, width, height, _p(None if pos is None else f32(pos)),
                              _p(None if look is None else f32(look)), y0, y1)
        film = np.zeros((height, width, 3), np.float32)
        lib().orc_get_film(self.h, _p(film))
        return film, int(ev)

    def encode(self, width: int, height: int, exposure: float, tonemap: bool = True):
        out = np.zeros((height, width, 3), np.uint8)
        lib().orc_encode(self.h, exposure, 1 if tonemap else 0, _p(out))
        return out


def srgb(c: float) -> int:
    return int(lib().orc_srgb(float(c)))


def form_factor_at(verts, p, n) -> float:
    v, p, n = f32(verts).reshape(12), f32(p), f32(n)
    return float(lib().orc_form_factor_at(_p(v), _p(p), _p(n)))


def camera_basis(pos, look, up, fov, w, h):
    out = np.zeros(14, np.float32)
    lib().orc_camera(_p(f32(pos)), _p(f32(look)), _p(f32(up)), fov, w, h, _p(out))
    return out


def counters(enable: bool, reset: bool = False):
    out = np.zeros(10, np.uint64)
    lib().orc_counters(1 if enable else 0, 1 if reset else 0, _p(out))
    return out
