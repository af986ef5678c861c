"""Collider authoring on the host: the brush record rule and the shape list DSL.

Restates, as host code producing `Brush` records for ``clay_volume_build_brushes``:
``BrushSet.make`` / ``compile`` (lib/src/field/brush.ts:407-438), the builtin reach rule
``builtinBound`` (brush.ts:183-217), ``eulerToQuat`` / ``quatMul`` (brush.ts:147-170), and
the list-folding shape DSL ``sdf.union`` / ``sdf.cut`` / ``Shape.at`` / ``smooth``
(lib/src/shape/sdf.ts:26-183). All arithmetic is JavaScript's binary64; the records are
rounded to f32 once, as the reference's buffer write does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

KINDS = {"sphere": 0, "box": 1, "roundBox": 2, "capsule": 3, "torus": 4, "cylinder": 5,
         "plane": 6, "boxFrame": 7, "volume": 8, "cone": 9, "octahedron": 10,
         "tetrahedron": 11, "dodecahedron": 12, "icosahedron": 13}
OPS = {"add": 0, "cut": 1, "paint": 2}

BRUSH_DTYPE = np.dtype([
    ("pos", np.float32, 3), ("scale", np.float32), ("rot", np.float32, 4),
    ("size", np.float32, 3), ("radius", np.float32), ("material", np.float32),
    ("blend", np.float32), ("bound", np.float32), ("mask", np.float32),
    ("kind", np.uint32), ("op", np.uint32), ("slot", np.uint32), ("pad", np.uint32),
])
assert BRUSH_DTYPE.itemsize == 80


def euler_to_quat(x: float, y: float, z: float):
    """brush.ts:147-157."""
    cx, sx = math.cos(x / 2), math.sin(x / 2)
    cy, sy = math.cos(y / 2), math.sin(y / 2)
    cz, sz = math.cos(z / 2), math.sin(z / 2)
    return (sx * cy * cz + cx * sy * sz, cx * sy * cz - sx * cy * sz,
            cx * cy * sz + sx * sy * cz, cx * cy * cz - sx * sy * sz)


def quat_mul(a, b):
    """Hamilton product, xyzw, `a` applied after `b` (brush.ts:160-170)."""
    return (a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1],
            a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0],
            a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3],
            a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2])


def normalize_size(size):
    if size is None:
        return (1.0, 1.0, 1.0)
    if isinstance(size, (int, float)):
        return (float(size),) * 3
    return (float(size[0]), float(size[1]), float(size[2]))


def builtin_bound(kind: str, size, radius: float) -> float:
    """Conservative reach of a builtin kind at unit scale (brush.ts:183-217)."""
    sx, sy, sz = size
    if kind == "sphere":
        return sx
    if kind in ("box", "boxFrame", "roundBox"):
        return math.hypot(sx, sy, sz) + radius
    if kind == "capsule":
        return sy + radius
    if kind == "torus":
        return sx + radius
    if kind == "cylinder":
        return math.hypot(sx, sy)
    if kind == "cone":
        return math.hypot(max(sx, sz), sy)
    if kind in ("octahedron", "tetrahedron", "dodecahedron", "icosahedron"):
        return sx
    if kind == "plane":
        return math.inf
    if kind == "volume":
        return sx * math.sqrt(3)
    raise ValueError(f"BrushSet: unknown primitive '{kind}'. Known: {', '.join(KINDS)}")


def make_brush(kind: str, op: str = "add", pos=None, euler=None, quat=None, scale=None,
               size=None, radius=None, material=None, smooth=None, onlyMaterial=None,
               slot=None, layer=None) -> np.ndarray:
    """BrushSet.make (brush.ts:407-430): one 80-byte record."""
    if kind not in KINDS:
        raise ValueError(f"BrushSet: unknown primitive '{kind}'. Known: {', '.join(KINDS)}")
    s = normalize_size(size)
    sc = 1.0 if scale is None else float(scale)
    r = 0.0 if radius is None else float(radius)
    sm = 0.02 if smooth is None else float(smooth)
    ex, ey, ez = euler if euler is not None else (0.0, 0.0, 0.0)
    bound = builtin_bound(kind, s, r) * sc + sm
    q = euler_to_quat(ex, ey, ez)
    if quat is not None:
        q = quat_mul(tuple(quat), q)
    rec = np.zeros(1, BRUSH_DTYPE)
    rec["pos"] = pos if pos is not None else (0.0, 0.0, 0.0)
    rec["scale"] = sc
    rec["rot"] = q
    rec["size"] = s
    rec["radius"] = r
    rec["material"] = 0.0 if material is None else float(material)
    rec["blend"] = sm
    rec["bound"] = bound if math.isfinite(bound) else 1e9
    rec["mask"] = -1.0 if onlyMaterial is None else float(onlyMaterial)
    rec["kind"] = KINDS[kind]
    rec["op"] = OPS[op]
    rec["slot"] = 0 if slot is None else int(slot)
    return rec


@dataclass(frozen=True)
class Node:
    kind: str
    op: str = "add"
    pos: tuple | None = None
    euler: tuple | None = None
    quat: tuple | None = None
    scale: float | None = None
    size: object = None
    radius: float | None = None
    material: float | None = None
    smooth: float | None = None
    onlyMaterial: float | None = None
    layer: int | None = None


@dataclass(frozen=True)
class Shape:
    """A brush list folded left to right (sdf.ts:26-83)."""

    nodes: tuple = field(default_factory=tuple)

    def _map(self, f):
        return Shape(tuple(f(n) for n in self.nodes))

    def at(self, pos):
        return self._map(lambda n: replace(n, pos=tuple((n.pos[i] if n.pos else 0.0) + pos[i]
                                                        for i in range(3))))

    def rotate(self, euler):
        return self._map(lambda n: replace(n, euler=tuple(euler)))

    def turn(self, q):
        return self._map(lambda n: replace(n, quat=tuple(q)))

    def scale(self, s):
        return self._map(lambda n: replace(n, scale=(n.scale if n.scale is not None else 1.0) * s))

    def material(self, m):
        return self._map(lambda n: n if n.material is not None else replace(n, material=m))

    def only(self, m):
        return self._map(lambda n: replace(n, onlyMaterial=m))

    def smooth(self, r):
        return self._map(lambda n: replace(n, smooth=r))


class sdf:
    """Primitives and CSG of sdf.ts:98-183."""

    @staticmethod
    def sphere(radius):
        return Shape((Node("sphere", size=radius),))

    @staticmethod
    def box(half):
        return Shape((Node("box", size=tuple(half)),))

    @staticmethod
    def roundBox(half, corner):
        return Shape((Node("roundBox", size=tuple(half), radius=corner),))

    @staticmethod
    def capsule(halfLength, radius):
        return Shape((Node("capsule", size=(0.0, halfLength, 0.0), radius=radius),))

    @staticmethod
    def torus(ring, tube):
        return Shape((Node("torus", size=ring, radius=tube),))

    @staticmethod
    def cylinder(radius, halfHeight):
        return Shape((Node("cylinder", size=(radius, halfHeight, radius)),))

    @staticmethod
    def cone(radius, halfHeight):
        return Shape((Node("cone", size=(radius, halfHeight, 0.0)),))

    @staticmethod
    def plane(y=0.0):
        return Shape((Node("plane", radius=y),))

    @staticmethod
    def union(*shapes):
        return Shape(tuple(n for s in shapes for n in s.nodes))

    @staticmethod
    def cut(a, *rest):
        out = list(a.nodes)
        for s in rest:
            for n in s.nodes:
                if n.op == "cut":
                    raise ValueError(
                        "sdf.cut: a subtraction inside a subtraction cannot be flattened into a "
                        "brush fold. Rewrite `cut(a, cut(b, c))` as a union of the pieces you want removed.")
                out.append(replace(n, op="paint" if n.op == "paint" else "cut"))
        return Shape(tuple(out))


def compile_shape(shape: Shape) -> np.ndarray:
    """compileShape + BrushSet.compile (sdf.ts:186-197, brush.ts:433-438): sorted by layer
    (stable), one record each."""
    order = sorted(range(len(shape.nodes)), key=lambda i: (shape.nodes[i].layer or 0, i))
    recs = [make_brush(n.kind, n.op, n.pos, n.euler, n.quat, n.scale, n.size, n.radius,
                       n.material, n.smooth, n.onlyMaterial) for n in (shape.nodes[i] for i in order)]
    if not recs:
        return np.zeros(0, BRUSH_DTYPE)
    return np.concatenate(recs)
