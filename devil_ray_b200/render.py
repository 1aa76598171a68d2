"""Host-side mirror of the reference's rendering classes on this path, over
the C-ABI:

  Camera        rendering/camera.hpp:18-118 (create_rays)
  ColorTable    color_table.hpp (add_point / add_alpha / sample, correct_opacity)
  ColorMap      color_map.hpp (samples, scalar_range)
  PointLight    rendering/point_light.hpp, default_light (renderer.cpp:141-159)
  Framebuffer   rendering/framebuffer.hpp:19-53 (clear, composite_background)
  Volume        rendering/volume.hpp:19-59 (field, samples, use_lighting,
                color_map, integrate, save-style compositing)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .api import UnstructuredMesh, _dev, _ptr, _stream

RAY_WORDS = 9          # dray::Ray: dir3, near, orig3, far, pixel_id
PARTIAL_WORDS = 6      # dray::VolumePartial: pixel, depth, rgba


class Camera:
    def __init__(self, width=500, height=500, pos=(0, 0, 0), look_at=(0, 0, -1), up=(0, 1, 0),
                 fov=30.0, zoom=1.0):
        self.width, self.height = width, height
        self.pos, self.look_at, self.up = pos, look_at, up
        self.fov, self.zoom = fov, zoom

    def desc(self) -> L.DrbCamera:
        c = L.DrbCamera()
        c.width, c.height = self.width, self.height
        for i in range(3):
            c.pos[i], c.look_at[i], c.up[i] = self.pos[i], self.look_at[i], self.up[i]
        c.fov_y, c.zoom = self.fov, self.zoom
        return c

    def _take(self, d: L.DrbCamera):
        self.pos = tuple(float(d.pos[i]) for i in range(3))
        self.look_at = tuple(float(d.look_at[i]) for i in range(3))
        self.fov = float(d.fov_y)

    def reset_to_bounds(self, bounds6, xpad=0.0, ypad=0.0, zpad=0.0):
        """Camera::reset_to_bounds: bounds6 = (xmin, xmax, ymin, ymax, zmin,
        zmax); look at their padded centre from the current direction, one
        diagonal away, with a 60-degree field of view."""
        d = self.desc()
        b = np.ascontiguousarray(bounds6, np.float32)
        L.check(L.lib().drb_camera_reset_to_bounds(C.byref(d), b.ctypes.data_as(C.c_void_p),
                                                   xpad, ypad, zpad),
                "drb_camera_reset_to_bounds")
        self._take(d)

    def elevate(self, degrees: float):
        d = self.desc()
        L.check(L.lib().drb_camera_elevate(C.byref(d), degrees), "drb_camera_elevate")
        self._take(d)

    def azimuth(self, degrees: float):
        d = self.desc()
        L.check(L.lib().drb_camera_azimuth(C.byref(d), degrees), "drb_camera_azimuth")
        self._take(d)

    def create_rays(self, device="cuda", stream=None, bounds=None) -> torch.Tensor:
        """Camera::create_rays (rays, bounds): the bounds argument is
        accepted and, as in the reference, not used."""
        n = self.width * self.height
        rays = torch.empty((n, RAY_WORDS), dtype=torch.float32, device=device)
        d = self.desc()
        L.check(L.lib().drb_camera_rays(C.byref(d), _ptr(rays), _stream(stream)),
                "drb_camera_rays")
        return rays


class PointLight:
    def __init__(self, pos=(0, 0, 0), amb=(0.4,) * 3, diff=(0.75,) * 3, spec=(0.8,) * 3,
                 spec_pow=15.0):
        self.pos, self.amb, self.diff, self.spec, self.spec_pow = pos, amb, diff, spec, spec_pow

    def as13(self):
        return np.array([*self.pos, *self.amb, *self.diff, *self.spec, self.spec_pow], np.float32)

    @staticmethod
    def default(camera: Camera) -> "PointLight":
        out = np.zeros(13, np.float32)
        d = camera.desc()
        L.check(L.lib().drb_default_light(C.byref(d), out.ctypes.data_as(C.c_void_p)),
                "drb_default_light")
        return PointLight(tuple(out[0:3]), tuple(out[3:6]), tuple(out[6:9]), tuple(out[9:12]),
                          float(out[12]))


def lights_tensor(lights, device):
    arr = np.stack([l.as13() for l in lights]) if lights else np.zeros((0, 13), np.float32)
    return torch.as_tensor(arr, device=device)


class ColorTable:
    def __init__(self, smooth=True):
        self.rgb = []      # (pos, r, g, b)
        self.alpha = []    # (pos, a)
        self.smooth = smooth

    def add_point(self, pos, rgb):
        self.rgb.append((float(pos), *map(float, rgb)))

    def add_alpha(self, pos, a):
        self.alpha.append((float(pos), float(a)))

    def sample(self, n, alpha_scale=1.0, opacity_factor=0.0) -> np.ndarray:
        out = np.zeros((n, 4), np.float32)
        rgb = np.array(self.rgb, np.float32).reshape(-1)
        al = np.array(self.alpha, np.float32).reshape(-1)
        L.check(L.lib().drb_color_table_sample(
            len(self.rgb), rgb.ctypes.data_as(C.c_void_p) if rgb.size else None,
            len(self.alpha), al.ctypes.data_as(C.c_void_p) if al.size else None,
            int(self.smooth), n, alpha_scale, opacity_factor, out.ctypes.data_as(C.c_void_p)),
            "drb_color_table_sample")
        return out


class ColorMap:
    def __init__(self, table: ColorTable | None = None, samples: int = 1024):
        self.table = table or ColorTable()
        self.n_samples = samples
        self.range = None

    def samples(self, n):
        self.n_samples = n

    def color_table(self, t: ColorTable):
        self.table = t

    def scalar_range(self, lo, hi):
        self.range = (float(lo), float(hi))


class UnstructuredField:
    """Scalar field on the mesh's element layout: UnstructuredField<HexScalar*>,
    or with shape=SHAPE_SIMPLEX UnstructuredField<TetScalar*>."""

    def __init__(self, ctrl_idx, values, order: int, name: str = "f", device="cuda",
                 shape: int = L.SHAPE_TENSOR):
        self.order = int(order)
        self.name = name
        self.shape = int(shape)
        self.device = torch.device(device)
        self.ctrl_idx = _dev(ctrl_idx, torch.int32, device)
        self.values = _dev(values, torch.float32, device).reshape(-1)
        nd = L.lib().drb_elem_dofs(self.shape, 3, self.order)
        if nd < 0:
            raise ValueError(f"unsupported field: shape {shape}, order {order}")
        self.n_elem = self.ctrl_idx.numel() // nd
        stride = L.lib().drb_packed_stride_shape(self.shape, 3, self.order, 1)
        self.packed = torch.empty((max(self.n_elem, 1), stride), dtype=torch.float32,
                                  device=self.device)
        d = self.desc(packed=False)
        L.check(L.lib().drb_pack_elements(C.byref(d), _ptr(self.packed), _stream(None)),
                "drb_pack_elements")
        self._range = None

    def desc(self, packed=True) -> L.DrbMesh:
        m = L.DrbMesh()
        m.dim, m.order, m.ncomp = 3, self.order, 1
        m.shape = self.shape
        m.n_elem = self.n_elem
        m.n_ctrl = self.values.numel()
        m.ctrl_idx = self.ctrl_idx.data_ptr()
        m.values = self.values.data_ptr()
        m.packed = self.packed.data_ptr() if packed else None
        return m

    def range(self):
        if self._range is None:
            r = torch.empty(2, dtype=torch.float32, device=self.device)
            d = self.desc()
            L.check(L.lib().drb_field_range(C.byref(d), _ptr(r), _stream(None)), "drb_field_range")
            self._range = tuple(float(x) for x in r.cpu())
        return self._range


class Framebuffer:
    def __init__(self, width, height, device="cuda"):
        self.width, self.height = width, height
        n = width * height
        self.colors = torch.zeros((n, 4), dtype=torch.float32, device=device)
        self.depths = torch.full((n,), float("inf"), dtype=torch.float32, device=device)
        self.bg_color = (1.0, 1.0, 1.0, 1.0)

    def clear(self, color=(0.0, 0.0, 0.0, 0.0), stream=None):
        c = np.array(color, np.float32)
        L.check(L.lib().drb_framebuffer_clear(_ptr(self.colors), _ptr(self.depths),
                                              self.width * self.height,
                                              c.ctypes.data_as(C.c_void_p), _stream(stream)),
                "drb_framebuffer_clear")

    def composite_background(self, stream=None):
        c = np.array(self.bg_color, np.float32)
        L.check(L.lib().drb_framebuffer_composite_background(
            _ptr(self.colors), self.width * self.height, c.ctypes.data_as(C.c_void_p),
            _stream(stream)), "drb_framebuffer_composite_background")

    def image(self) -> np.ndarray:
        return self.colors.reshape(self.height, self.width, 4).cpu().numpy()


def cull_rays(rays: torch.Tensor, bounds6, stream=None) -> torch.Tensor:
    """remove_missed_rays: active rays with near/far from the slab test."""
    n = rays.shape[0]
    out = torch.empty_like(rays)
    b = np.array(bounds6, np.float32)
    na = C.c_int()
    L.check(L.lib().drb_cull_rays(_ptr(rays), n, b.ctypes.data_as(C.c_void_p), _ptr(out),
                                  C.byref(na), _stream(stream)), "drb_cull_rays")
    return out[: na.value]


class Volume:
    """Volume renderer over one mesh + scalar field (single domain)."""

    def __init__(self, mesh: UnstructuredMesh, field: UnstructuredField):
        self.mesh, self.field_ = mesh, field
        if mesh.dim == 3:
            mesh.face_neighbors()  # the march steps across element faces with them
        self.n_samples = 100
        self.lighting = True
        self.cmap = ColorMap()
        # Volume() adds these alphas to its default table (volume.cpp:277-281)
        self.cmap.table.add_alpha(0.1, 0.0)
        self.cmap.table.add_alpha(1.0, 0.7)
        self.tol, self.max_steps = 1e-4, 20
        self.guess_mode = L.GUESS_ELEM_CENTER
        self.coherent = False
        self._tf_cache = None

    def samples(self, n):
        self.n_samples = int(n)

    def use_lighting(self, on: bool):
        self.lighting = bool(on)

    def color_map(self) -> ColorMap:
        return self.cmap

    def _opts(self) -> L.DrbVolumeOpts:
        o = L.DrbVolumeOpts()
        o.samples, o.use_lighting = self.n_samples, int(self.lighting)
        o.tol, o.max_steps = self.tol, self.max_steps
        o.guess_mode, o.coherent = self.guess_mode, int(self.coherent)
        b = self.mesh.bounds()
        for i in range(6):
            o.bounds[i] = float(b[i])
        return o

    # integrate_partials samples the opacity-corrected table into a freshly
    # constructed ColorMap, whose sample count is the default 1024 whatever
    # the user's ColorMap::samples (volume.cpp:81-87, color_map.cpp:11-17)
    TF_SAMPLES = 1024

    def _tf(self):
        key = (self.n_samples, tuple(self.cmap.table.rgb), tuple(self.cmap.table.alpha),
               self.cmap.table.smooth)
        if self._tf_cache is None or self._tf_cache[0] != key:
            # correct_opacity(10 / samples) then ColorMap sampling (volume.cpp:81-87)
            tf = self.cmap.table.sample(self.TF_SAMPLES, 1.0, 10.0 / self.n_samples)
            self._tf_cache = (key, torch.as_tensor(tf, device=self.mesh.device))
        return self._tf_cache[1]

    def _range(self):
        r = self.cmap.range or self.field_.range()
        return np.array(r, np.float32)

    def integrate(self, rays: torch.Tensor, lights, stats=False, stream=None):
        """Volume::integrate: compacted partials [n, 6] (pixel as float bits)."""
        active = cull_rays(rays, self.mesh.bounds(), stream)
        n = active.shape[0]
        parts = torch.empty((max(5 * n, 1), PARTIAL_WORDS), dtype=torch.float32,
                            device=self.mesh.device)
        lt = lights_tensor(lights, self.mesh.device)
        o = self._opts()
        tf = self._tf()
        rng = self._range()
        np_ = C.c_int()
        st, rs = self._stats(n, stats)
        bd = self.mesh.get_bvh().desc()  # first: it may add the mesh's hull planes
        L.check(L.lib().drb_volume_integrate(
            C.byref(self.mesh.desc()), C.byref(self.field_.desc()),
            C.byref(bd), _ptr(active), n, C.byref(o), _ptr(tf),
            tf.shape[0], rng.ctypes.data_as(C.c_void_p), _ptr(lt), len(lights), _ptr(parts),
            C.byref(np_), rs, _stream(stream)), "drb_volume_integrate")
        out = parts[: np_.value]
        return (out, st) if stats else out

    def _stats(self, n, stats):
        if not stats:
            return None, L.DrbRayStats()
        st = [torch.zeros(max(n, 1), dtype=torch.int32, device=self.mesh.device) for _ in range(3)]
        return st, L.DrbRayStats(*(t.data_ptr() for t in st))

    def render(self, camera: Camera, lights=None, fb: Framebuffer | None = None, stats=False,
               stream=None, active=None):
        """Rays -> cull -> fused integrate+composite -> Framebuffer (before
        the background composite)."""
        if lights is None:
            lights = [PointLight.default(camera)]
        if fb is None:
            fb = Framebuffer(camera.width, camera.height, self.mesh.device)
        fb.clear(stream=stream)
        if active is None:
            rays = camera.create_rays(self.mesh.device, stream)
            active = cull_rays(rays, self.mesh.bounds(), stream)
        n = active.shape[0]
        lt = lights_tensor(lights, self.mesh.device)
        o = self._opts()
        tf = self._tf()
        rng = self._range()
        st, rs = self._stats(n, stats)
        bd = self.mesh.get_bvh().desc()  # first: it may add the mesh's hull planes
        L.check(L.lib().drb_volume_render(
            C.byref(self.mesh.desc()), C.byref(self.field_.desc()),
            C.byref(bd), _ptr(active), n, C.byref(o), _ptr(tf),
            tf.shape[0], rng.ctypes.data_as(C.c_void_p), _ptr(lt), len(lights),
            _ptr(fb.colors), _ptr(fb.depths), rs, _stream(stream)), "drb_volume_render")
        return (fb, st) if stats else fb

    def save_image(self, partials: torch.Tensor, width, height, stream=None) -> Framebuffer:
        """Volume::save compositing (without the PNG): partials -> framebuffer
        with the white background composited."""
        fb = Framebuffer(width, height, self.mesh.device)
        fb.clear(stream=stream)
        L.check(L.lib().drb_composite_partials(_ptr(partials), partials.shape[0],
                                               _ptr(fb.colors), _stream(stream)),
                "drb_composite_partials")
        fb.composite_background(stream)
        return fb


class MeshBoundary:
    """MeshBoundary::execute for one hex or tet mesh (+ scalar field): the
    boundary quad (or triangle) mesh and face field sharing the volume's
    value arrays."""

    def execute(self, mesh: UnstructuredMesh, field: UnstructuredField | None = None,
                stream=None):
        d = mesh.desc()
        nf = C.c_int()
        L.check(L.lib().drb_mesh_boundary(C.byref(d), None, None, None, None, C.byref(nf),
                                          _stream(stream)), "drb_mesh_boundary")
        p = mesh.order
        n = nf.value
        dev = mesh.device
        shape = getattr(mesh, "shape", L.SHAPE_TENSOR)
        nd2 = L.lib().drb_elem_dofs(shape, 2, p)
        fidx = torch.empty((max(n, 1), nd2), dtype=torch.int32, device=dev)
        ffidx = torch.empty_like(fidx) if field is not None else None
        elface = torch.empty((max(n, 1), 2), dtype=torch.int32, device=dev)
        L.check(L.lib().drb_mesh_boundary(C.byref(d),
                                          None if field is None else _ptr(field.ctrl_idx),
                                          _ptr(fidx), _ptr(ffidx), _ptr(elface), C.byref(nf),
                                          _stream(stream)), "drb_mesh_boundary")
        faces = UnstructuredMesh(fidx[:n].reshape(-1), mesh.dof_data.values, p, dim=2, device=dev,
                                 shape=shape)
        face_field = None
        if field is not None:
            face_field = QuadField(ffidx[:n].reshape(-1), field.values, p, name=field.name,
                                   device=dev, shape=shape)
        self.elid_faceid = elface[:n]
        return faces, face_field


class QuadField(UnstructuredField):
    """Scalar field on the faces of a 2D mesh: UnstructuredField<QuadScalar*>,
    or with shape=SHAPE_SIMPLEX UnstructuredField<TriScalar*>."""

    def __init__(self, ctrl_idx, values, order: int, name: str = "f", device="cuda",
                 shape: int = L.SHAPE_TENSOR):
        self.order = int(order)
        self.name = name
        self.shape = int(shape)
        self.device = torch.device(device)
        self.ctrl_idx = _dev(ctrl_idx, torch.int32, device)
        self.values = _dev(values, torch.float32, device).reshape(-1)
        nd = L.lib().drb_elem_dofs(self.shape, 2, self.order)
        self.n_elem = self.ctrl_idx.numel() // nd
        stride = L.lib().drb_packed_stride_shape(self.shape, 2, self.order, 1)
        self.packed = torch.empty((max(self.n_elem, 1), stride), dtype=torch.float32,
                                  device=self.device)
        d = self.desc(packed=False)
        L.check(L.lib().drb_pack_elements(C.byref(d), _ptr(self.packed), _stream(None)),
                "drb_pack_elements")
        self._range = None

    def desc(self, packed=True) -> L.DrbMesh:
        m = super().desc(packed)
        m.dim = 2
        return m


class Surface:
    """Surface of a quad or triangle mesh (Surface / Traceable)."""

    def __init__(self, faces: UnstructuredMesh, field: UnstructuredField):
        self.faces, self.field_ = faces, field
        self.cmap = ColorMap()
        self.tol, self.max_steps = 1e-4, 10   # face_intersection.hpp:153-154

    def color_map(self) -> ColorMap:
        return self.cmap

    def nearest_hit(self, rays: torch.Tensor, stats=False, stream=None):
        n = rays.shape[0]
        hits = torch.empty((n, 5), dtype=torch.float32, device=self.faces.device)
        st = [torch.zeros(max(n, 1), dtype=torch.int32, device=self.faces.device)
              for _ in range(2)] if stats else None
        rs = L.DrbRayStats(None, *(t.data_ptr() for t in st)) if stats else L.DrbRayStats()
        L.check(L.lib().drb_surface_intersect(C.byref(self.faces.desc()),
                                              C.byref(self.faces.get_bvh().desc()), _ptr(rays),
                                              n, self.tol, self.max_steps, _ptr(hits), rs,
                                              _stream(stream)), "drb_surface_intersect")
        return (hits, st) if stats else hits

    def _tf(self):
        return torch.as_tensor(self.cmap.table.sample(self.cmap.n_samples), device=self.faces.device)

    def shade(self, rays, hits, lights, fb: Framebuffer, use_lighting=True, stream=None):
        n = rays.shape[0]
        frags = torch.empty((n, 4), dtype=torch.float32, device=self.faces.device)
        tf = self._tf()
        rng = np.array(self.cmap.range or self.field_.range(), np.float32)
        lt = lights_tensor(lights, self.faces.device)
        L.check(L.lib().drb_surface_shade(C.byref(self.faces.desc()), C.byref(self.field_.desc()),
                                          _ptr(rays), _ptr(hits), n, _ptr(tf), tf.shape[0],
                                          rng.ctypes.data_as(C.c_void_p), _ptr(lt), len(lights),
                                          int(use_lighting), _ptr(frags), _ptr(fb.colors),
                                          _ptr(fb.depths), _stream(stream)), "drb_surface_shade")
        return frags

    def render(self, camera: Camera, lights=None, use_lighting=True, stream=None):
        if lights is None:
            lights = [PointLight.default(camera)]
        rays = camera.create_rays(self.faces.device, stream)
        fb = Framebuffer(camera.width, camera.height, self.faces.device)
        fb.clear(stream=stream)
        hits = self.nearest_hit(rays, stream=stream)
        self.shade(rays, hits, lights, fb, use_lighting, stream)
        return fb, hits


class ScalarBuffer:
    """ScalarBuffer (rendering/scalar_buffer.cpp): per-pixel depth, zone id
    and one plane per field, cleared to clear_value (zone ids to -1)."""

    def __init__(self, width, height, clear_value=float("nan"), device="cuda"):
        self.width, self.height, self.clear_value = width, height, clear_value
        self.device = torch.device(device)
        n = width * height
        self.depths = torch.full((n,), clear_value, dtype=torch.float32, device=self.device)
        self.zone_ids = torch.full((n,), -1, dtype=torch.int32, device=self.device)
        self.scalars: dict[str, torch.Tensor] = {}

    def has_field(self, name):
        return name in self.scalars

    def add_field(self, name):
        self.scalars[name] = torch.full((self.width * self.height,), self.clear_value,
                                        dtype=torch.float32, device=self.device)


class ScalarRenderer:
    """ScalarRenderer (rendering/scalar_renderer.cpp:296-462) over one
    surface: the nearest hit of every camera ray, its depth and zone id, and
    the value of each named field at the hit, per pixel (no colour map)."""

    def __init__(self, surface: Surface, fields: dict):
        self.surface = surface
        self.fields = dict(fields)     # name -> face field on the surface's quads
        self.names: list[str] = []

    def field_names(self, names):
        self.names = list(names)

    def render(self, camera: Camera, stream=None) -> ScalarBuffer:
        rays = camera.create_rays(self.surface.faces.device, stream)
        buf = ScalarBuffer(camera.width, camera.height, device=self.surface.faces.device)
        self.render_rays(rays, buf, stream)
        return buf

    def render_rays(self, rays, buf: ScalarBuffer, stream=None):
        n = rays.shape[0]
        dev = self.surface.faces.device
        hits = self.surface.nearest_hit(rays, stream=stream)
        L.check(L.lib().drb_scalar_buffer_write(_ptr(rays), _ptr(hits), None, n, 0,
                                                _ptr(buf.depths), _ptr(buf.zone_ids), None,
                                                _stream(stream)), "drb_scalar_buffer_write")
        tf = torch.zeros((1, 4), dtype=torch.float32, device=dev)
        rng = np.zeros(2, np.float32)
        for name in self.names:
            if name not in self.fields:
                continue
            frags = torch.empty((n, 4), dtype=torch.float32, device=dev)
            L.check(L.lib().drb_surface_shade(C.byref(self.surface.faces.desc()),
                                              C.byref(self.fields[name].desc()), None, _ptr(hits),
                                              n, _ptr(tf), 1, rng.ctypes.data_as(C.c_void_p),
                                              None, 0, 0, _ptr(frags), None, None,
                                              _stream(stream)), "drb_surface_shade")
            if not buf.has_field(name):
                buf.add_field(name)
            L.check(L.lib().drb_scalar_buffer_write(_ptr(rays), _ptr(hits), _ptr(frags), n, 0,
                                                    None, None, _ptr(buf.scalars[name]),
                                                    _stream(stream)), "drb_scalar_buffer_write")
        L.check(L.lib().drb_ray_max(_ptr(rays), _ptr(hits), n, _stream(stream)), "drb_ray_max")
        return buf


class PointLocation:
    """PointLocation (queries/point_location.cpp:178-287), one domain: field
    values at arbitrary points, the empty value where no element holds the
    point.  Locates with the reference's settings (tol 1e-4, 20 steps)
    through the batched kernel, then evaluates each field on the device."""

    def __init__(self):
        self.vars: list[str] = []
        self.empty = 0.0
        self.tol, self.max_steps, self.guess_mode = 1e-4, 20, L.GUESS_ELEM_CENTER

    def add_var(self, name: str):
        self.vars.append(name)

    def empty_val(self, v: float):
        self.empty = float(v)

    def execute(self, mesh: UnstructuredMesh, fields: dict, points, stream=None):
        from .api import BatchedLocator
        pts = _dev(points, torch.float32, mesh.device).reshape(-1, 3)
        loc = BatchedLocator(mesh, self.tol, self.max_steps, self.guess_mode)
        cell, ref = loc.locate(pts, stream=stream)
        out = {}
        for v in self.vars:
            if v not in fields:
                continue
            f = fields[v]
            vals = torch.empty(pts.shape[0], dtype=torch.float32, device=mesh.device)
            L.check(L.lib().drb_field_eval(C.byref(f.desc()), _ptr(cell), _ptr(ref),
                                           pts.shape[0], self.empty, _ptr(vals),
                                           _stream(stream)), "drb_field_eval")
            out[v] = vals
        return out


class Lineout:
    """Lineout (queries/lineout.cpp): field values at samples + 2 evenly
    spaced points along each line, start and end included."""

    def __init__(self):
        self.n_samples = 100
        self.empty = 0.0
        self.starts, self.ends, self.vars = [], [], []
        self.locator = PointLocation()

    def samples(self, n: int):
        if n < 1:
            raise ValueError("Number of samples must be positive")
        self.n_samples = int(n)

    def empty_val(self, v: float):
        self.empty = float(v)

    def add_line(self, start, end):
        self.starts.append(tuple(float(x) for x in start))
        self.ends.append(tuple(float(x) for x in end))

    def add_var(self, name: str):
        self.vars.append(name)

    def create_points(self, device, stream=None):
        a = torch.tensor(self.starts, dtype=torch.float32, device=device).reshape(-1, 3)
        b = torch.tensor(self.ends, dtype=torch.float32, device=device).reshape(-1, 3)
        pts = torch.empty((a.shape[0] * (self.n_samples + 2), 3), dtype=torch.float32,
                          device=device)
        L.check(L.lib().drb_lineout_points(_ptr(a), _ptr(b), a.shape[0], self.n_samples,
                                           _ptr(pts), _stream(stream)), "drb_lineout_points")
        return pts

    def execute(self, mesh: UnstructuredMesh, fields: dict, stream=None):
        """(points [n_lines * (samples + 2), 3], {var: values})."""
        if not self.vars:
            raise ValueError("Lineout: must specify at least 1 variables:")
        if not self.starts:
            raise ValueError("Lineout: must specify at least 1 line:")
        if not any(v in fields for v in self.vars):
            raise ValueError("Lineout: must specify at least one valid field.")
        pts = self.create_points(mesh.device, stream)
        self.locator.vars = list(self.vars)
        self.locator.empty_val(self.empty)
        return pts, self.locator.execute(mesh, fields, pts, stream)
