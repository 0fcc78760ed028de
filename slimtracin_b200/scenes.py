"""Seeded synthetic scenes in the reference's struct layout.

One generator feeds the device path, the oracle and the reference harness with the same bytes.
PCG32 (O'Neill 2014, XSH-RR output) with seed 0x5EED0000 + config drives every draw; rotations are
uniform unit quaternions by Shoemake's method.  No public dataset is involved.

Scenes (sizes as the benchmark uses them; tests use the size arguments to shrink them):
  implicit16_scene  16 implicit primitives (4 each of sphere/box/quad/tetrahedron), 3 point
                    lights, Lambert/Blinn/Phong materials, 640x480, depth 2.
  mesh_scene        one displaced icosphere mesh (subdivision 8 = 1,310,720 triangles) in 8
                    instances, 4 Cook-Torrance + 2 glass + 2 mirror materials with 1024^2
                    albedo/normal textures, 2 emissive quads, 1920x1080, depth 4.
  moving_scene      4096 implicit primitives moving every frame, 1280x720, depth 2.

The reference has no shininess field: the Blinn/Phong exponent is {16,4}*(1-roughness)
(render/shaders/common.h:294-316), so "shininess U[2,128]" maps to roughness U[0, 0.875].
"""
from dataclasses import dataclass, field
import ctypes as C

import numpy as np

from . import structs as S

F32 = np.float32


class PCG32:
    """PCG32 XSH-RR, 64-bit state, default increment."""
    MULT = 6364136223846793005
    INC = 1442695040888963407
    MASK = (1 << 64) - 1

    def __init__(self, seed):
        self.state = 0
        self.next_u32()
        self.state = (self.state + seed) & self.MASK
        self.next_u32()

    def next_u32(self):
        old = self.state
        self.state = (old * self.MULT + self.INC) & self.MASK
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, lo=0.0, hi=1.0, n=None):
        if n is None:
            return lo + (hi - lo) * (self.next_u32() / 4294967296.0)
        return np.array([self.uniform(lo, hi) for _ in range(n)], dtype=np.float64)

    def quaternion(self):
        """Shoemake's uniform random rotation; returns (x, y, z, w)."""
        u1, u2, u3 = self.uniform(), self.uniform(), self.uniform()
        a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
        return np.array([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                         b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)])

    def numpy_rng(self):
        return np.random.default_rng(self.next_u32() | (self.next_u32() << 32))


# ------------------------------------------------------------------------------------------------
# quaternion helpers (float64); the convention is the reference's mulVec3Quat (math/quat.h:25):
# v' = v + 2w(a x v) + 2 a x (a x v) for q = (a, w)
def quat_to_matrix_cols(q):
    x, y, z, w = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def matrix_cols_to_quat(m):
    t = np.trace(m)
    if t > 0:
        s = np.sqrt(t + 1.0) * 2
        w, x, y, z = 0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = np.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2
        w, x, y, z = (m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s
    elif m[1, 1] > m[2, 2]:
        s = np.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2
        w, x, y, z = (m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s
    else:
        s = np.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2
        w, x, y, z = (m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s
    q = np.array([x, y, z, w])
    return q / np.linalg.norm(q)


def rot_x(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])


def rot_y(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


# ------------------------------------------------------------------------------------------------
@dataclass
class CameraSpec:
    """A pinhole camera: position, yaw (about +y) and pitch (about +x, positive looks down)."""
    position: tuple = (0.0, 0.0, -15.0)
    yaw: float = 0.0
    pitch: float = 0.0
    focal_length: float = 2.0

    def matrix_cols(self):
        # view -> world; columns are right, up, forward
        return rot_y(self.yaw) @ rot_x(self.pitch)


def look_at(position, target, focal_length=2.0):
    d = np.asarray(target, dtype=np.float64) - np.asarray(position, dtype=np.float64)
    d /= np.linalg.norm(d)
    yaw = np.arctan2(d[0], d[2])
    pitch = -np.arcsin(d[1])
    return CameraSpec(tuple(position), float(yaw), float(pitch), focal_length)


def fill_camera(cam: S.Camera, spec: CameraSpec):
    """Fill a reference Camera struct (core/types.h:169) from a CameraSpec."""
    C.memset(C.addressof(cam), 0, C.sizeof(cam))
    m = spec.matrix_cols()
    minv = m.T
    cam.focal_length = cam.zoom = F32(spec.focal_length)
    cam.target_distance = 10
    t = cam.transform
    ident = np.eye(3)
    for name in ("matrix", "yaw_matrix", "pitch_matrix", "roll_matrix"):
        _set_mat3(getattr(t, name), ident)
    _set_mat3(t.rotation_matrix, m)
    _set_mat3(t.rotation_matrix_inverted, minv)
    _set_quat(t.rotation, matrix_cols_to_quat(m))
    _set_quat(t.rotation_inverted, matrix_cols_to_quat(minv))
    t.position.x, t.position.y, t.position.z = [F32(v) for v in spec.position]
    t.scale.x = t.scale.y = t.scale.z = 1
    t.right_direction = C.pointer(t.rotation_matrix.X)
    t.up_direction = C.pointer(t.rotation_matrix.Y)
    t.forward_direction = C.pointer(t.rotation_matrix.Z)


def _set_mat3(dst, m_cols):
    # the reference's mat3 rows X, Y, Z are the columns of the view->world matrix
    for row, col in zip((dst.X, dst.Y, dst.Z), m_cols.T):
        row.x, row.y, row.z = [F32(v) for v in col]


def _set_quat(dst, q):
    dst.axis.x, dst.axis.y, dst.axis.z, dst.amount = [F32(v) for v in q]


def set_projection_plane(vp: S.Viewport, cam: S.Camera, grid_w: int, grid_h: int):
    """setViewportProjectionPlane (core/init.h:545) for a QCAA frame buffer, in float32 with the
    reference's operation order (no fused operations), so the plane is bit-identical to the one
    the reference's beginDrawing computes."""
    R = cam.transform.rotation_matrix
    fwd = np.array([R.Z.x, R.Z.y, R.Z.z], dtype=F32)
    right_dir = np.array([R.X.x, R.X.y, R.X.z], dtype=F32)
    up = np.array([R.Y.x, R.Y.y, R.Y.z], dtype=F32)
    f_height = F32(grid_h)
    offset = F32(0.0)
    start = fwd * F32(f_height * F32(cam.focal_length))
    right = right_dir * F32(offset - F32(grid_w))
    down = up * F32(f_height - offset)
    start = start + right
    start = start + down
    right = right_dir * F32(2)
    down = up * F32(-2)
    pp = vp.projection_plane
    pp.start.x, pp.start.y, pp.start.z = [F32(v) for v in start]
    pp.right.x, pp.right.y, pp.right.z = [F32(v) for v in right]
    pp.down.x, pp.down.y, pp.down.z = [F32(v) for v in down]


def set_projection_matrix(vp: S.Viewport, cam: S.Camera, dim: S.Dimensions):
    """setProjectionMatrix (viewport/viewport.h:95) in float32: the matrix beginDrawing leaves in
    viewport->projection_matrix, which the debug overlays project their edges with."""
    n = F32(vp.settings.near_clipping_plane_distance)
    f = F32(vp.settings.far_clipping_plane_distance)
    fl = F32(cam.focal_length)
    ar = F32(dim.height_over_width)
    gl = bool(vp.settings.use_cube_NDC)
    M = vp.projection_matrix
    for row in (M.X, M.Y, M.Z, M.W):
        row.x = row.y = row.z = row.w = 0.0
    M.Z.w = 1.0
    M.X.x = F32(fl * ar)
    M.Y.y = fl
    zz = F32(F32(1.0) / F32(f - n))
    M.Z.z = F32(zz * (F32(f + n) if gl else f))
    M.W.z = F32(zz * (F32(F32(F32(-2) * f) * n) if gl else F32(F32(-n) * f)))


def update_dimensions(dim: S.Dimensions, width, height, qcaa=True):
    """updateDimensions (core/base.h:344)."""
    if qcaa:
        width += 1
        height += 1
    dim.width, dim.height = width, height
    dim.width_times_height = width * height
    dim.f_width, dim.f_height = F32(width), F32(height)
    dim.h_width = F32(F32(width) / F32(2))
    dim.h_height = F32(F32(height) / F32(2))
    dim.width_over_height = F32(F32(width) / F32(height))
    dim.height_over_width = F32(F32(height) / F32(width))


class Frame:
    """A Viewport + Camera + PixelGrid + output buffers for one view (reference structs)."""

    def __init__(self, width, height, camera: CameraSpec, depth=2, mode=S.RM_BEAUTY, cone_angle=0.0,
                 with_pixels=True, with_float=True):
        self.width, self.height = width, height
        self.grid_w, self.grid_h = width + 1, height + 1
        self.camera = S.Camera()
        fill_camera(self.camera, camera)
        self.grid = S.PixelGrid()
        update_dimensions(self.grid.dimensions, width, height, True)
        self.grid.QCAA = 1
        self.float_pixels = np.zeros(self.grid_w * self.grid_h, dtype=S.FLOATPIXEL_DT) if with_float else None
        self.pixels = np.zeros(width * height, dtype=S.PIXEL_DT) if with_pixels else None
        self.grid.float_pixels = self.float_pixels.ctypes.data if with_float else None
        self.grid.pixels = self.pixels.ctypes.data if with_pixels else None
        self.viewport = S.Viewport()
        vp = self.viewport
        vp.camera = C.pointer(self.camera)
        vp.frame_buffer = C.pointer(self.grid)
        s = vp.settings
        s.near_clipping_plane_distance = F32(0.001)
        s.far_clipping_plane_distance = F32(1000.0)
        s.background_opacity = 1.0
        s.render_mode = mode
        s.background_fill = 1
        s.antialias = 1
        s.use_GPU = 1
        vp.trace.depth = depth
        set_projection_plane(vp, self.camera, self.grid_w, self.grid_h)
        set_projection_matrix(vp, self.camera, self.grid.dimensions)
        vp.projection_plane.cone_angle = F32(cone_angle)

    @property
    def rays(self):
        return self.grid_w * self.grid_h


# ------------------------------------------------------------------------------------------------
@dataclass
class TextureData:
    width: int
    height: int
    wrap: bool
    mipmap: bool
    mips: list  # [(w, h, TexelQuad array of (w+1)*(h+1))]


@dataclass
class MeshData:
    positions: np.ndarray          # (V,3) f32
    normals: np.ndarray            # (V,3) f32
    uvs: np.ndarray                # (V,2) f32
    indices: np.ndarray            # (T,3) u32 position indices
    aabb: np.ndarray               # (6,) f32 min, max
    triangles: np.ndarray = None   # (T,) TRIANGLE_DT, BVH-ordered
    nodes: np.ndarray = None       # (2T,) BVHNODE_DT
    leaf_ids: np.ndarray = None    # (T,) u32
    node_count: int = 0
    height: int = 0
    normal_indices: np.ndarray = None  # (T,3) u32; None -> the position indices
    uv_indices: np.ndarray = None      # (T,3) u32; None -> the position indices

    @property
    def triangle_count(self):
        return len(self.indices)

    def allocate_bvh(self):
        t = self.triangle_count
        self.triangles = np.zeros(t, dtype=S.TRIANGLE_DT)
        self.nodes = np.zeros(max(2 * t, 1), dtype=S.BVHNODE_DT)
        self.leaf_ids = np.zeros(max(t, 1), dtype=np.uint32)

    def to_ctypes(self, keep):
        m = S.Mesh()
        m.aabb.min.x, m.aabb.min.y, m.aabb.min.z = [F32(v) for v in self.aabb[:3]]
        m.aabb.max.x, m.aabb.max.y, m.aabb.max.z = [F32(v) for v in self.aabb[3:]]
        m.triangle_count = self.triangle_count
        m.vertex_count = len(self.positions)
        m.normals_count = len(self.normals)
        m.uvs_count = len(self.uvs)
        m.edge_count = 0
        nidx = self.indices if self.normal_indices is None else self.normal_indices
        uidx = self.indices if self.uv_indices is None else self.uv_indices
        for name, arr in (("vertex_positions", self.positions), ("vertex_normals", self.normals),
                          ("vertex_uvs", self.uvs), ("vertex_position_indices", self.indices),
                          ("vertex_normal_indices", nidx), ("vertex_uvs_indices", uidx)):
            arr = np.ascontiguousarray(arr)
            keep.append(arr)
            setattr(m, name, arr.ctypes.data)
        if self.triangles is None:
            self.allocate_bvh()
        m.triangles = self.triangles.ctypes.data
        m.bvh.nodes = self.nodes.ctypes.data
        m.bvh.leaf_ids = self.leaf_ids.ctypes.data
        m.bvh.node_count = self.node_count
        m.bvh.height = self.height
        return m

    def read_back(self, m):
        self.node_count = m.bvh.node_count
        self.height = m.bvh.height


@dataclass
class SceneData:
    primitives: np.ndarray
    materials: np.ndarray
    lights: np.ndarray
    ambient: tuple = (0.0, 0.0, 0.0)
    meshes: list = field(default_factory=list)
    textures: list = field(default_factory=list)
    tlas_nodes: np.ndarray = None
    tlas_leaf_ids: np.ndarray = None
    tlas_node_count: int = 0
    tlas_height: int = 0
    name: str = ""

    def __post_init__(self):
        if self.tlas_nodes is None:
            n = len(self.primitives)
            self.tlas_nodes = np.zeros(max(2 * n, 1), dtype=S.BVHNODE_DT)
            self.tlas_leaf_ids = np.zeros(max(n, 1), dtype=np.uint32)

    def copy(self):
        import copy
        c = copy.copy(self)
        c.primitives = self.primitives.copy()
        c.tlas_nodes = self.tlas_nodes.copy()
        c.tlas_leaf_ids = self.tlas_leaf_ids.copy()
        return c

    def to_ctypes(self):
        """Build a reference Scene struct over this data.  Returns (scene, keepalive)."""
        keep = []
        sc = S.Scene()
        st = sc.settings
        st.cameras = 1
        st.primitives = len(self.primitives)
        st.materials = len(self.materials)
        st.lights = len(self.lights)
        st.meshes = len(self.meshes)
        st.textures = len(self.textures)
        sc.ambient_light.x, sc.ambient_light.y, sc.ambient_light.z = [F32(v) for v in self.ambient]
        for name, arr in (("primitives", self.primitives), ("materials", self.materials),
                          ("lights", self.lights)):
            if len(arr):
                setattr(sc, name, arr.ctypes.data)
        if self.meshes:
            meshes = (S.Mesh * len(self.meshes))()
            for i, md in enumerate(self.meshes):
                meshes[i] = md.to_ctypes(keep)
            counts = np.array([md.node_count for md in self.meshes], dtype=np.uint32)
            tris = np.array([md.triangle_count for md in self.meshes], dtype=np.uint32)
            keep += [meshes, counts, tris]
            sc.meshes = C.addressof(meshes)
            sc.mesh_bvh_node_counts = counts.ctypes.data
            sc.mesh_triangle_counts = tris.ctypes.data
        if self.textures:
            texs = (S.Texture * len(self.textures))()
            for i, td in enumerate(self.textures):
                mips = (S.TextureMip * len(td.mips))()
                for j, (w, h, quads) in enumerate(td.mips):
                    mips[j].width, mips[j].height = w, h
                    mips[j].texel_quads = quads.ctypes.data
                keep.append(mips)
                texs[i].width, texs[i].height = td.width, td.height
                texs[i].mip_count = len(td.mips)
                texs[i].wrap, texs[i].mipmap = int(td.wrap), int(td.mipmap)
                texs[i].mips = C.cast(mips, C.POINTER(S.TextureMip))
            keep.append(texs)
            sc.textures = C.addressof(texs)
        sc.bvh.nodes = self.tlas_nodes.ctypes.data
        sc.bvh.leaf_ids = self.tlas_leaf_ids.ctypes.data
        sc.bvh.node_count = self.tlas_node_count
        sc.bvh.height = self.tlas_height
        return sc, keep

    def read_back_tlas(self, sc):
        self.tlas_node_count = sc.bvh.node_count
        self.tlas_height = sc.bvh.height


def default_materials(n):
    """initMaterial (core/init.h:478) for n materials."""
    m = np.zeros(n, dtype=S.MATERIAL_DT)
    m["reflectivity"] = 1
    m["albedo"] = 1
    m["roughness"] = 1
    m["n1_over_n2"] = 1
    m["n2_over_n1"] = 1
    m["uv_repeat"] = 1
    m["brdf"] = S.BRDF_LAMBERT
    m["use"] = S.NORMAL_MAP | S.ALBEDO_MAP
    return m


def default_primitives(n):
    """initPrimitive (core/init.h:461) with id = index (app.h:186)."""
    p = np.zeros(n, dtype=S.PRIMITIVE_DT)
    p["color"] = 1
    p["flags"] = S.ALL_FLAGS
    p["scale"] = 1
    p["rotation"][:, 3] = 1
    p["id"] = np.arange(n)
    return p


def default_lights(n):
    """initScene's light defaults (app.h:160-168)."""
    lt = np.zeros(n, dtype=S.LIGHT_DT)
    lt["color"] = 1
    lt["attenuation"] = 1
    lt["intensity"] = 1
    return lt


# ------------------------------------------------------------------------------------------------
_IMPLICIT_TYPES = (S.PT_SPHERE, S.PT_BOX, S.PT_QUAD, S.PT_TETRAHEDRON)


def _random_implicit(rng: PCG32, n, blocks=True):
    prims = default_primitives(n)
    for i in range(n):
        prims["type"][i] = _IMPLICIT_TYPES[(i * 4 // n) if blocks else (rng.next_u32() % 4)]
        prims["position"][i] = rng.uniform(-5, 5, 3)
        prims["scale"][i] = rng.uniform(0.3, 1.5, 3)
        prims["rotation"][i] = rng.quaternion()
    return prims


def _classic_materials(rng: PCG32, n):
    mats = default_materials(n)
    brdfs = (S.BRDF_LAMBERT, S.BRDF_BLINN, S.BRDF_PHONG)
    for i in range(n):
        mats["brdf"][i] = brdfs[i % 3]
        mats["albedo"][i] = rng.uniform(0, 1, 3)
        mats["roughness"][i] = rng.uniform(0, 0.875)
    return mats


def _point_lights(rng: PCG32, n):
    lights = default_lights(n)
    for i in range(n):
        lights["intensity"][i] = rng.uniform(1, 10)
        lights["position_or_direction"][i] = (rng.uniform(-8, 8), rng.uniform(4, 10), rng.uniform(-8, 8))
    return lights


def implicit16_scene(seed_offset=0):
    """16 implicit primitives (4 of each type in blocks), 3 point lights, 16 classic materials."""
    rng = PCG32(0x5EED0000 + 0 + seed_offset)
    prims = _random_implicit(rng, 16, blocks=True)
    prims["material_id"] = np.arange(16)
    mats = _classic_materials(rng, 16)
    lights = _point_lights(rng, 3)
    sd = SceneData(prims, mats, lights, ambient=(0.004, 0.004, 0.007), name="implicit16")
    return sd, CameraSpec((0.0, 0.0, -15.0), 0.0, 0.0, 2.0)


def moving_scene(seed_offset=0, count=4096, spread=5.0):
    """`count` implicit primitives of uniformly drawn types, same distributions as implicit16_scene, plus
    per-primitive velocities (units/frame) and angular velocities (axis, rad/frame)."""
    rng = PCG32(0x5EED0000 + 2 + seed_offset)
    prims = default_primitives(count)
    vel = np.zeros((count, 3))
    ang = np.zeros((count, 4))
    for i in range(count):
        prims["type"][i] = _IMPLICIT_TYPES[rng.next_u32() % 4]
        prims["position"][i] = rng.uniform(-spread, spread, 3)
        prims["scale"][i] = rng.uniform(0.3, 1.5, 3)
        prims["rotation"][i] = rng.quaternion()
        vel[i] = rng.uniform(-0.5, 0.5, 3)
        axis = rng.quaternion()[:3]
        ang[i, :3] = axis / max(np.linalg.norm(axis), 1e-12)
        ang[i, 3] = rng.uniform(0, 0.05)
    mats = _classic_materials(rng, 16)
    prims["material_id"] = np.arange(count) % 16
    lights = _point_lights(rng, 3)
    sd = SceneData(prims, mats, lights, ambient=(0.004, 0.004, 0.007), name="moving")
    sd.velocities = vel
    sd.angular = ang
    return sd, CameraSpec((0.0, 0.0, -15.0 - spread), 0.0, 0.0, 2.0)


def advance_moving_scene(sd: SceneData, frames=1):
    """Integrate the moving scene's motion by `frames` steps in float32 on the host."""
    p = sd.primitives
    for _ in range(frames):
        p["position"] = (p["position"] + sd.velocities.astype(F32)).astype(F32)
        half = sd.angular[:, 3] * 0.5
        dq = np.concatenate([sd.angular[:, :3] * np.sin(half)[:, None], np.cos(half)[:, None]], 1)
        q = p["rotation"].astype(np.float64)
        x1, y1, z1, w1 = dq.T
        x2, y2, z2, w2 = q.T
        out = np.stack([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                        w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                        w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2,
                        w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2], 1)
        out /= np.linalg.norm(out, axis=1, keepdims=True)
        p["rotation"] = out.astype(F32)


# ------------------------------------------------------------------------------------------------
def icosphere(subdivisions):
    """Unit icosphere: 20 * 4^s triangles, 10 * 4^s + 2 shared vertices."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                      [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                     dtype=np.float64)
    faces = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                      [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                      [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                      [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    for _ in range(subdivisions):
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        edges = np.concatenate([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)])
        edges.sort(axis=1)
        key = edges[:, 0] * (len(verts) + 1) + edges[:, 1]
        uniq, inverse = np.unique(key, return_inverse=True)
        e0, e1 = uniq // (len(verts) + 1), uniq % (len(verts) + 1)
        mid = verts[e0] + verts[e1]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(verts)
        verts = np.concatenate([verts, mid])
        nf = len(faces)
        ab = base + inverse[:nf]
        bc = base + inverse[nf:2 * nf]
        ca = base + inverse[2 * nf:]
        faces = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                                np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return verts, faces


def value_noise3(p, rng_seed, frequency=4.0, octaves=3):
    """Seeded 3D value noise (trilinear over a hashed lattice, smoothstep fade)."""
    rng = np.random.default_rng(rng_seed)
    table = rng.random(4096)
    perm = rng.permutation(4096)
    out = np.zeros(len(p))
    amp, freq, norm = 1.0, frequency, 0.0
    for _ in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        f = f * f * (3 - 2 * f)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    h = perm[(perm[(perm[(i0[:, 0] + dx) & 4095] + i0[:, 1] + dy) & 4095] + i0[:, 2] + dz) & 4095]
                    w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2])
                    acc += w * table[h]
        out += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2
    return out / norm * 2 - 1


def displaced_icosphere(subdivisions, seed, amplitude=0.1, radius=1.0):
    """Icosphere with vertices displaced along the normal by value noise; area-weighted vertex
    normals; spherical UVs; centred on its AABB like obj2mesh does (obj2mesh.c:25)."""
    v, f = icosphere(subdivisions)
    v = radius * v * (1.0 + amplitude * value_noise3(v, seed))[:, None]
    e1 = v[f[:, 1]] - v[f[:, 0]]
    e2 = v[f[:, 2]] - v[f[:, 0]]
    fn = np.cross(e1, e2)  # length = 2 * area: area weighting
    vn = np.zeros_like(v)
    for k in range(3):
        np.add.at(vn, f[:, k], fn)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    d = v / np.linalg.norm(v, axis=1, keepdims=True)
    uv = np.stack([0.5 + np.arctan2(d[:, 2], d[:, 0]) / (2 * np.pi), 0.5 - np.arcsin(np.clip(d[:, 1], -1, 1)) / np.pi], 1)
    lo, hi = v.min(0), v.max(0)
    v = v - (lo + hi) / 2
    v32 = v.astype(F32)
    aabb = np.concatenate([v32.min(0), v32.max(0)]).astype(F32)
    return MeshData(v32, vn.astype(F32), uv.astype(F32), f.astype(np.uint32), aabb)


# ------------------------------------------------------------------------------------------------
def perlin2(width, height, seed, cells=8, octaves=4):
    """Seeded tileable 2D gradient (Perlin) noise in [0,1], shape (height, width)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((height, width))
    amp, norm = 1.0, 0.0
    ys, xs = np.mgrid[0:height, 0:width]
    for o in range(octaves):
        n = cells * (2 ** o)
        ang = rng.random((n, n)) * 2 * np.pi
        gx, gy = np.cos(ang), np.sin(ang)
        px, py = xs * n / width, ys * n / height
        x0, y0 = np.floor(px).astype(int), np.floor(py).astype(int)
        fx, fy = px - x0, py - y0
        acc = 0
        for dx in (0, 1):
            for dy in (0, 1):
                ix, iy = (x0 + dx) % n, (y0 + dy) % n
                dot = gx[iy, ix] * (fx - dx) + gy[iy, ix] * (fy - dy)
                wx = 6 * fx ** 5 - 15 * fx ** 4 + 10 * fx ** 3
                wy = 6 * fy ** 5 - 15 * fy ** 4 + 10 * fy ** 3
                acc = acc + dot * (wx if dx else 1 - wx) * (wy if dy else 1 - wy)
        out += amp * acc
        norm += amp
        amp *= 0.5
    return np.clip(out / norm * 1.2 + 0.5, 0, 1)


def perlin_textures(size, seed):
    """(albedo RGB, normal-map RGB) uint8 images of size x size from seeded Perlin noise."""
    h = perlin2(size, size, seed)
    h2 = perlin2(size, size, seed + 1, cells=4)
    albedo = np.stack([0.25 + 0.7 * h, 0.2 + 0.6 * h2, 0.15 + 0.5 * (1 - h)], -1)
    gy, gx = np.gradient(h * 8.0)
    n = np.stack([-gx, -gy, np.ones_like(h)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    normal = (n * 0.5 + 0.5)
    return ((albedo * 255).astype(np.uint8), (normal * 255).astype(np.uint8))


def _quad_sources(w, h, wrap):
    """Which texel each quadrant of each (w+1)x(h+1) texel quad ends up holding after
    loadTextureMipLoader (bmp2texture.c:181-237): index arrays (qy, qx) -> texel (ty, tx) for the
    quadrants TL, TR, BL, BR.  Clamp mode clamps both axes.  Wrap mode wraps every axis except the
    right-hand quadrants of the last quad column, which the loop overwrites with clamped values
    after wrapping them (so only its bottom-row BR and top-row TR corners keep the wrapped texel)."""
    qy, qx = np.mgrid[0:h + 1, 0:w + 1]
    left_x = qx - 1
    right_x = qx.copy()
    top_y = qy - 1
    bottom_y = qy.copy()
    if wrap:
        left_x = np.where(qx == 0, w - 1, left_x)
        top_y = np.where(qy == 0, h - 1, top_y)
        bottom_y = np.where(qy == h, 0, bottom_y)
        right_tr = np.where(qx == w, np.where(qy == 0, 0, w - 1), right_x)
        right_br = np.where(qx == w, np.where(qy == h, 0, w - 1), right_x)
    else:
        left_x = np.maximum(left_x, 0)
        top_y = np.maximum(top_y, 0)
        bottom_y = np.minimum(bottom_y, h - 1)
        right_tr = right_br = np.minimum(right_x, w - 1)
    return {"TL": (top_y, left_x), "TR": (top_y, right_tr), "BL": (bottom_y, left_x),
            "BR": (bottom_y, right_br)}


def bake_texture(rgb, wrap=True, mipmap=True):
    """loadTexture (bmp2texture.c:324): float texels, TexelQuad grids with the reference's edge
    replication, box-filtered mips down to 4 px (summed TL+TR+BL+BR in that order, times 0.25, in
    float32), truncated to u8 at the end."""
    height, width = rgb.shape[:2]
    texels = rgb[..., :3].astype(F32)
    mips = []
    w, h = width, height
    while True:
        src = _quad_sources(w, h, wrap)
        quads = np.zeros((h + 1) * (w + 1), dtype=S.TEXELQUAD_DT)
        for k, name in enumerate(("TL", "TR", "BL", "BR")):
            ty, tx = src[name]
            vals = texels[ty, tx].reshape(-1, 3)
            quads["R"][:, k] = vals[:, 0].astype(np.uint8)
            quads["G"][:, k] = vals[:, 1].astype(np.uint8)
            quads["B"][:, k] = vals[:, 2].astype(np.uint8)
        mips.append((w, h, quads))
        if not (mipmap and w > 4 and h > 4):
            break
        mw, mh = w // 2, h // 2
        tl = texels[0:2 * mh:2, 0:2 * mw:2]
        tr = texels[0:2 * mh:2, 1:2 * mw:2]
        bl = texels[1:2 * mh:2, 0:2 * mw:2]
        br = texels[1:2 * mh:2, 1:2 * mw:2]
        texels = (((tl + tr) + bl) + br) * F32(0.25)
        w, h = mw, mh
    return TextureData(width, height, wrap, mipmap, mips)


def mesh_scene(seed_offset=0, subdivisions=8, texture_size=1024, instances=8, radius=2.5):
    """The 1080p PBR mesh scene (sizes at the defaults).  The icosphere has radius 2.5 and the camera
    frames the instances (about 42% of primary rays hit, 27% a mesh instance at 1080p); neither is
    fixed by the benchmark's description."""
    rng = PCG32(0x5EED0000 + 1 + seed_offset)
    mesh = displaced_icosphere(subdivisions, seed=rng.next_u32(), radius=radius)
    n_prims = instances + 2
    prims = default_primitives(n_prims)
    for i in range(instances):
        prims["type"][i] = S.PT_MESH
        prims["id"][i] = 0
        prims["position"][i] = (rng.uniform(-8, 8), rng.uniform(0, 4), rng.uniform(-8, 8))
        prims["rotation"][i] = rng.quaternion()
        prims["scale"][i] = rng.uniform(0.5, 1.5, 3)
        prims["material_id"][i] = i
    # two emissive quads placed as in examples/06_AreaLights.c:170-188
    h2 = F32(0.70710678118)
    for j, (x, rot_w) in enumerate(((-15.0, h2), (15.0, -h2))):
        k = instances + j
        prims["type"][k] = S.PT_QUAD
        prims["position"][k] = (x, 5.0, 5.0)
        prims["rotation"][k] = (0.0, 0.0, -h2, rot_w)
        prims["scale"][k] = (4.0, 1.0, 8.0)
        prims["material_id"][k] = instances + j
    mats = default_materials(instances + 2)
    for i in range(instances):
        m = mats[i]
        m["texture_count"] = 2
        m["texture_ids"][:2] = (0, 1)
        m["use"] = S.ALBEDO_MAP | S.NORMAL_MAP
        m["uv_repeat"] = (2.0, 2.0)
        kind = i % 4
        if i < 4:
            m["brdf"] = S.BRDF_COOK_TORRANCE
            m["roughness"] = rng.uniform(0.05, 1.0)
            metallic = 1.0 if rng.uniform() < 0.3 else 0.0
            m["metallic"] = metallic
            alb = rng.uniform(0, 1, 3)
            m["albedo"] = alb
            m["reflectivity"] = 0.04 + (alb - 0.04) * metallic
        elif i < 6:
            m["is_"] = S.REFRACTIVE
            m["brdf"] = S.BRDF_BLINN
            m["roughness"] = 0.0
            m["n1_over_n2"] = F32(S.IOR_AIR / F32(1.5))
            m["n2_over_n1"] = F32(F32(1.5) / S.IOR_AIR)
            m["albedo"] = (0.9, 0.95, 1.0)
        else:
            m["is_"] = S.REFLECTIVE
            m["brdf"] = S.BRDF_PHONG
            m["roughness"] = 0.1
            m["reflectivity"] = 0.9
        del kind
    for j, em in enumerate(((0.9, 0.7, 0.7), (0.7, 0.7, 0.9))):
        mats[instances + j]["is_"] = S.EMISSIVE
        mats[instances + j]["emission"] = em
    albedo, normal = perlin_textures(texture_size, seed=rng.next_u32())
    textures = [bake_texture(albedo, True, True), bake_texture(normal, True, True)]
    sd = SceneData(prims, mats, default_lights(0), ambient=(0.004, 0.004, 0.007),
                   meshes=[mesh], textures=textures, name="mesh")
    cam = look_at((0.0, 8.0, -15.0), (0.0, 1.5, 0.0))
    return sd, cam


# ------------------------------------------------------------------------------------------------
def example_area_lights():
    """examples/06_AreaLights.c setupScene (:142-199): floor, two emissive quads, two spheres,
    three point lights (a scene with both point lights and emissive quads)."""
    prims = default_primitives(5)
    FLOOR, L1, L2, S1, S2 = range(5)
    prims["type"][[S1, S2]] = S.PT_SPHERE
    prims["type"][[FLOOR, L1, L2]] = S.PT_QUAD
    prims["material_id"][L1], prims["material_id"][L2] = 1, 2
    h2 = F32(0.70710678118)
    prims["rotation"][L1] = (0, 0, -h2, h2)
    prims["rotation"][L2] = (0, 0, -h2, -h2)
    prims["position"][S1] = (3, 3, 0)
    prims["position"][S2] = (-3, 3, 0)
    prims["position"][L1] = (-15, 5, 5)
    prims["position"][L2] = (15, 5, 5)
    prims["scale"][FLOOR] = (40, 1, 40)
    prims["scale"][L1] = (4, 1, 8)
    prims["scale"][L2] = (4, 1, 8)
    mats = default_materials(3)
    mats["is_"][1] = mats["is_"][2] = S.EMISSIVE
    mats["emission"][1] = (0.9, 0.7, 0.7)
    mats["emission"][2] = (0.7, 0.7, 0.9)
    mats["albedo"][0] = (0.8, 1.0, 0.8)
    lights = default_lights(3)
    lights["intensity"] = (F32(1.1) * F32(40), F32(1.2) * F32(40), F32(0.9) * F32(40))
    lights["color"] = ((1, 1, 0.65), (1, 0.25, 0.25), (0.65, 0.65, 1))
    lights["position_or_direction"] = ((10, 10, -5), (2, 5, 12), (-10, 10, -5))
    sd = SceneData(prims, mats, lights, ambient=(0.004, 0.004, 0.007), name="06_AreaLights")
    return sd, CameraSpec((0.0, 7.0, -11.0), 0.0, 0.2, 2.0)
