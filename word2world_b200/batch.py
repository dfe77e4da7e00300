"""Batched rendering: many views of many scenes with one launch per stage.

The reference renders one view per call (``Renderer.render`` ->
``rasterize_gaussians`` / ``rasterize_gaussians_backward``).  A batch here is a
list of items, each one view (camera, resolution, background) of one scene
(its activated parameter tensors, resident on the device); the whole batch is
projected, culled, scanned, keyed, sorted, blended and back-propagated with
one launch per stage through the C ABI's ``w2w_batch_*`` entry points
(include/w2w_raster.h).  Each item's image equals what a single-view call
returns for it (bit-identical), and its gradients equal the single-view
call's up to the order of float atomic additions.

Keys are (global tile, depth): one sort serves every item, and every tile's
list is exactly the list its item alone would produce, including the
reference's key-emission spill (the instance scan restarts its spill
component at every item).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _C  # noqa: F401  (loads libw2w_raster.so through the binding; also fails loudly when unbuilt)
from .camera import Camera

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libw2w_raster.so")
_lib = None

GRAD_MODES = {"reference": 0, "exact": 1}


class _Item(ctypes.Structure):
    _fields_ = [("means3D", ctypes.c_void_p), ("scales", ctypes.c_void_p), ("rotations", ctypes.c_void_p),
                ("opacities", ctypes.c_void_p), ("shs", ctypes.c_void_p),
                ("P", ctypes.c_int), ("M", ctypes.c_int), ("degree", ctypes.c_int), ("width", ctypes.c_int),
                ("height", ctypes.c_int),
                ("focal_x", ctypes.c_float), ("tan_fovx", ctypes.c_float), ("tan_fovy", ctypes.c_float),
                ("scale_modifier", ctypes.c_float),
                ("viewmatrix", ctypes.c_float * 16), ("projmatrix", ctypes.c_float * 16),
                ("campos", ctypes.c_float * 3), ("background", ctypes.c_float * 3)]


class _Info(ctypes.Structure):
    _fields_ = [("num_rendered", ctypes.c_longlong), ("depth_min_bits", ctypes.c_uint32),
                ("depth_max_bits", ctypes.c_uint32), ("error", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(_LIB_PATH)
        for fn in ("w2w_batch_geometry_state_bytes", "w2w_batch_image_state_bytes",
                   "w2w_batch_binning_state_bytes", "w2w_batch_backward_scratch_bytes"):
            getattr(L, fn).restype = ctypes.c_size_t
        L.w2w_batch_binning_state_bytes.argtypes = [ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int]
        L.w2w_status_string.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().w2w_status_string(rc).decode()} (status {rc})")


@dataclass
class Scene:
    """Activated parameters of one scene, resident on the device (the
    reference's ``Renderer.render`` inputs after its activation preamble)."""
    means3D: torch.Tensor     # [P,3]
    opacities: torch.Tensor   # [P,1]
    scales: torch.Tensor      # [P,3]
    rotations: torch.Tensor   # [P,4] (w, x, y, z)
    shs: torch.Tensor         # [P,M,3]
    sh_degree: int = 3

    @property
    def P(self) -> int:
        return int(self.means3D.shape[0])

    @classmethod
    def from_ply(cls, path, device="cuda", sh_degree: int = 3) -> "Scene":
        """A resident scene from a PLY file in the reference's layout
        (``ply.save_ply``), activated as ``Renderer.render`` activates."""
        from .ply import load_ply
        d = load_ply(path)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)
        opac, scales, rots, shs = _C.activate(t(d["opacity"]), t(d["svec"]), t(d["quaternion"]), t(d["sh_dc"]),
                                              t(d["sh_ac"]))
        return cls(t(d["mean"]), opac, scales, rots, shs, sh_degree)

    @classmethod
    def from_arrays(cls, arrays, device, sh_degree: int = 3) -> "Scene":
        m, o, s, q, sh = arrays
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)
        return cls(t(m), t(o), t(s), t(q), t(sh), sh_degree)


@dataclass
class View:
    scene: int                 # index into the batch's scene list
    camera: Camera
    background: tuple = (1.0, 1.0, 1.0)


@dataclass
class BatchResult:
    """Forward outputs of a batch; ``color[v]`` etc. are views into the
    packed buffers."""
    color: list
    depth: list
    alpha: list
    radii: list
    num_rendered: int
    state: dict = field(repr=False, default_factory=dict)


class _Workspace:
    """Grow-only device buffers, one per role, reused from call to call.

    Batches of different sizes would otherwise ask the caching allocator for
    new multi-GB blocks of ever different sizes; when its cache cannot serve
    one it synchronises and returns memory to the driver before retrying,
    which stalls a serving loop for tens of milliseconds.  Here a role's
    buffer is replaced only when a call needs more than it holds, by twice
    the need, so a growing stream of batches settles after a few growths; the
    old buffer goes back to the driver before the new one is taken, so the
    cache never holds dead blocks of old sizes."""

    def __init__(self, device):
        self.device = device
        self.bufs = {}
        self.grown = 0

    def take(self, role: str, nbytes: int) -> torch.Tensor:
        need = int(nbytes)
        b = self.bufs.get(role)
        if b is None or b.numel() < need:
            if self.bufs.pop(role, None) is not None and self.device.type == "cuda":
                del b
                torch.cuda.empty_cache()
            size = (max(2 * need, 256) + 255) // 256 * 256
            b = torch.empty(size, dtype=torch.uint8, device=self.device)
            self.bufs[role] = b
            self.grown += 1
        return b[:need]

    def f32(self, role: str, *shape) -> torch.Tensor:
        n = int(np.prod(shape))
        return self.take(role, 4 * n).view(torch.float32).view(*shape)

    def i32(self, role: str, n: int) -> torch.Tensor:
        return self.take(role, 4 * n).view(torch.int32)

    def i64(self, role: str, n: int) -> torch.Tensor:
        return self.take(role, 8 * n).view(torch.int64)

    @property
    def bytes(self) -> int:
        return sum(b.numel() for b in self.bufs.values())


class BatchRenderer:
    """Forward + backward of a list of (scene, view) items, one launch per stage.

    With ``reuse_buffers`` every device buffer of a call (state, images,
    gradients) comes from a grow-only workspace owned by the renderer, so a
    stream of batches of varying size makes no allocator calls once the
    workspace has grown to the largest batch.  A forward's outputs are then
    valid until the next forward, a backward's until the next backward."""

    def __init__(self, grad_mode: str = "reference", compat_spill: bool = True, device=None,
                 reuse_buffers: bool = False):
        self.grad_mode = GRAD_MODES[grad_mode]
        self.compat_spill = int(bool(compat_spill))
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.ws = _Workspace(self.device) if reuse_buffers else None

    def _pinned_tables(self, nbytes: int) -> torch.Tensor:
        """Grow-only pinned host buffer for the group tables; before it is
        refilled, the previous call's copy out of it has finished."""
        ev = getattr(self, "_tables_copied", None)
        if ev is not None:
            ev.synchronize()
        buf = getattr(self, "_pinned", None)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(2 * int(nbytes), 4096), dtype=torch.uint8).pin_memory()
            self._pinned = buf
        return buf

    def _u8(self, role, nbytes):
        if self.ws is not None:
            return self.ws.take(role, nbytes)
        return torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)

    def _f32(self, role, *shape):
        if self.ws is not None:
            return self.ws.f32(role, *shape)
        return torch.empty(*shape, dtype=torch.float32, device=self.device)

    def _i32(self, role, n):
        if self.ws is not None:
            return self.ws.i32(role, n)
        return torch.empty(n, dtype=torch.int32, device=self.device)

    # ---- item table -------------------------------------------------------
    def _items(self, scenes, views):
        n = len(views)
        arr = (_Item * n)()
        M = None
        for v, view in enumerate(views):
            sc = scenes[view.scene]
            for name in ("means3D", "opacities", "scales", "rotations", "shs"):
                t = getattr(sc, name)
                if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                    raise ValueError(f"scene {view.scene}: {name} must be a contiguous float32 CUDA tensor")
            m = int(sc.shs.shape[1])
            if M is None:
                M = m
            elif m != M:
                raise ValueError("all scenes of a batch need the same number of SH coefficients")
            cam = view.camera
            it = arr[v]
            it.means3D, it.scales, it.rotations = sc.means3D.data_ptr(), sc.scales.data_ptr(), sc.rotations.data_ptr()
            it.opacities, it.shs = sc.opacities.data_ptr(), sc.shs.data_ptr()
            it.P, it.M, it.degree = sc.P, m, int(sc.sh_degree)
            it.width, it.height = int(cam.width), int(cam.height)
            it.focal_x = float(cam.focal_x)
            it.tan_fovx, it.tan_fovy = float(cam.tanfovx), float(cam.tanfovy)
            it.scale_modifier = 1.0
            it.viewmatrix[:] = [float(x) for x in np.asarray(cam.viewmatrix, np.float32).reshape(-1)]
            it.projmatrix[:] = [float(x) for x in np.asarray(cam.projmatrix, np.float32).reshape(-1)]
            it.campos[:] = [float(x) for x in np.asarray(cam.campos, np.float32).reshape(-1)]
            it.background[:] = [float(x) for x in view.background]
        return arr, M

    @staticmethod
    def layout(views):
        """First pixel of every item in the packed per-pixel buffers (colour:
        three times that), and the total pixel count."""
        pb, p = [], 0
        for v in views:
            pb.append(p)
            p += int(v.camera.width) * int(v.camera.height)
        return pb, p

    # ---- forward ------------------------------------------------------------
    def forward(self, scenes, views) -> BatchResult:
        L = lib()
        arr, M = self._items(scenes, views)
        n = len(views)
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        E = sum(scenes[v.scene].P for v in views)
        dev = self.device
        geom = self._u8("geom", int(L.w2w_batch_geometry_state_bytes(arr, n)))
        radii = self._i32("radii", max(E, 1))
        info = _Info()
        _check(L.w2w_batch_forward_geometry(arr, n, self.compat_spill, ctypes.c_void_p(radii.data_ptr()),
                                            ctypes.c_void_p(geom.data_ptr()), ctypes.byref(info), stream),
               "batch forward geometry")
        R = int(info.num_rendered)
        binb = self._u8("binb", max(int(L.w2w_batch_binning_state_bytes(R, arr, n)), 1))
        img = self._u8("img", int(L.w2w_batch_image_state_bytes(arr, n)))
        pbase, npix = self.layout(views)
        color = self._f32("color", 3 * npix)
        depth = self._f32("depth", npix)
        alpha = self._f32("alpha", npix)
        _check(L.w2w_batch_forward_render(arr, n, ctypes.c_void_p(geom.data_ptr()), ctypes.byref(info),
                                          ctypes.c_void_p(binb.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                                          ctypes.c_void_p(color.data_ptr()), ctypes.c_void_p(depth.data_ptr()),
                                          ctypes.c_void_p(alpha.data_ptr()), stream), "batch forward render")
        cols, deps, alps, rads = [], [], [], []
        e = 0
        for v, view in enumerate(views):
            H, W = int(view.camera.height), int(view.camera.width)
            p = pbase[v]
            cols.append(color[3 * p:3 * p + 3 * H * W].view(3, H, W))
            deps.append(depth[p:p + H * W].view(1, H, W))
            alps.append(alpha[p:p + H * W].view(1, H, W))
            P = scenes[view.scene].P
            rads.append(radii[e:e + P])
            e += P
        state = dict(arr=arr, n=n, M=M, E=E, R=R, geom=geom, binb=binb, img=img, radii=radii, alpha=alpha,
                     npix=npix, pbase=pbase, scenes=scenes, views=views)
        return BatchResult(cols, deps, alps, rads, R, state)

    # ---- backward -----------------------------------------------------------
    def backward(self, res: BatchResult, dL_dcolor, dL_ddepth=None, dL_dalpha=None, per_element: bool = False,
                 groups=None, grouped: bool = True):
        """Gradients for upstream image gradients given per item (lists of
        [3,H,W] / [1,H,W] tensors).  Items are summed by group (default: by
        scene; a serving loop groups by request): returns, per group, the sum
        over its items of dL/d(means3D, opacity, scales, rotations, shs), in
        order of first appearance (``out["groups"]`` lists the group ids),
        plus the per-item dL/dmeans2D; ``per_element`` also returns the raw
        per-item tensors (the single-view call's eight outputs for every
        item).  Without ``per_element`` the per-Gaussian pass sums each
        group's items itself (w2w_batch_backward_grouped); ``grouped=False``
        writes per-item gradients and sums them with w2w_group_sum instead
        (the same sums in the same order, up to a few ulps)."""
        L = lib()
        st = res.state
        arr, n, M, E, R = st["arr"], st["n"], st["M"], st["E"], st["R"]
        dev = self.device
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        views, scenes = st["views"], st["scenes"]
        def packed(role, gs):
            out = self._f32(role, 3 * st["npix"] if role == "dlc" else st["npix"])
            torch.cat([g.reshape(-1) for g in gs], out=out)
            return out
        dlc = packed("dlc", dL_dcolor)
        # absent depth / alpha gradients go to the library as null (read as
        # zero; without both, the per-pixel backward leaves their terms out)
        dld = packed("dld", dL_ddepth) if dL_ddepth is not None else None
        dla = packed("dla", dL_dalpha) if dL_dalpha is not None else None
        scratch = self._u8("scratch", int(L.w2w_batch_backward_scratch_bytes(arr, n)))
        # the groups' tables (w2w_group_sum's layout): row bases, item pointers, item element bases
        gid = [groups[v] if groups is not None else views[v].scene for v in range(n)]
        order, base, total, members = [], {}, 0, {}
        ebase, e0 = [], 0
        for v in range(n):
            P = scenes[views[v].scene].P
            ebase.append(e0)
            e0 += P
            g = gid[v]
            if g not in base:
                base[g] = total
                order.append(g)
                members[g] = []
                total += P
            elif scenes[views[members[g][0]].scene].P != P:
                raise ValueError(f"group {g!r} mixes scenes of different sizes")
            members[g].append(v)
        size = {g: scenes[views[members[g][0]].scene].P for g in order}
        G = len(order)
        tab = np.empty(2 * (G + 1) + n, dtype=np.uint32)
        tab[:G] = [base[g] for g in order]
        tab[G] = total
        ptr, items = [0], []
        for g in order:
            items += [ebase[v] for v in members[g]]
            ptr.append(len(items))
        tab[G + 1:2 * (G + 1)] = ptr
        tab[2 * (G + 1):] = items
        tables = self._u8("group_tables", tab.nbytes)
        # from pinned memory without blocking the host: a copy from pageable
        # memory would wait for the backward kernels queued before it, so a
        # serving loop could not launch its next batch meanwhile
        staged = self._pinned_tables(tab.nbytes)
        staged[:tab.nbytes].copy_(torch.from_numpy(tab.view(np.uint8)))
        tables.copy_(staged[:tab.nbytes], non_blocking=True)
        self._tables_copied = torch.cuda.Event()
        self._tables_copied.record(torch.cuda.current_stream(dev))
        Eg = max(E, 1)
        f = self._f32
        g_m2, g_col, g_op = f("g_m2", Eg, 3), f("g_col", Eg, 3), f("g_op", Eg, 1)
        p = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else None)
        shapes = (("means3D", (3,)), ("opacities", (1,)), ("scales", (3,)), ("rotations", (4,)),
                  ("shs", (max(M, 1), 3)))
        out = {"groups": order}
        if grouped and not per_element:
            acc = {name: f("acc_" + name, max(total, 1), *shp) for name, shp in shapes}
            _check(L.w2w_batch_backward_grouped(
                arr, n, p(st["geom"]), ctypes.c_longlong(R), p(st["binb"]), p(st["img"]), p(st["radii"]),
                p(st["alpha"]), p(dlc), p(dld), p(dla), self.grad_mode, p(scratch), ctypes.c_size_t(scratch.numel()),
                p(tables), G, ctypes.c_longlong(total), p(g_m2), p(g_col), p(g_op), p(acc["means3D"]),
                p(acc["opacities"]), p(acc["scales"]), p(acc["rotations"]), p(acc["shs"]), stream),
                "batch backward (grouped)")
            for name, _ in shapes:
                out[name] = [acc[name][base[g]:base[g] + size[g]] for g in order]
        else:
            g_m3, g_cov, g_sh = f("g_m3", Eg, 3), f("g_cov", Eg, 6), f("g_sh", Eg, max(M, 1), 3)
            g_sc, g_rot = f("g_sc", Eg, 3), f("g_rot", Eg, 4)
            _check(L.w2w_batch_backward(arr, n, p(st["geom"]), ctypes.c_longlong(R), p(st["binb"]), p(st["img"]),
                                        p(st["radii"]), p(st["alpha"]), p(dlc), p(dld), p(dla), self.grad_mode,
                                        p(scratch), ctypes.c_size_t(scratch.numel()), p(g_m2), p(g_col), p(g_op),
                                        p(g_m3), p(g_cov), p(g_sh), p(g_sc), p(g_rot), stream), "batch backward")
            # per-group sums of the items' element ranges: one deterministic
            # reduction launch per tensor (w2w_group_sum)
            for name, t in (("means3D", g_m3), ("opacities", g_op), ("scales", g_sc), ("rotations", g_rot),
                            ("shs", g_sh)):
                width = int(np.prod(t.shape[1:]))
                acc_t = self._f32("acc_" + name, total, *t.shape[1:])
                _check(L.w2w_group_sum(p(t), width, G, p(tables), n, p(acc_t), ctypes.c_longlong(total), stream),
                       "group sum")
                out[name] = [acc_t[base[g]:base[g] + size[g]] for g in order]
        # the per-element accumulators and tables of this call (a grouped pass
        # can be re-run over them: w2w_batch_gaussians_grouped)
        self._last_backward = dict(scratch=scratch, g_m2=g_m2, g_col=g_col, g_op=g_op, tables=tables, G=G,
                                   total=total)
        e = 0
        out["means2D"] = []
        raw = []
        for v in views:
            P = scenes[v.scene].P
            out["means2D"].append(g_m2[e:e + P])
            if per_element:
                raw.append((g_m2[e:e + P], g_col[e:e + P], g_op[e:e + P], g_m3[e:e + P], g_cov[e:e + P],
                            g_sh[e:e + P], g_sc[e:e + P], g_rot[e:e + P]))
            e += P
        if per_element:
            out["per_item"] = raw
        return out
