"""A double-precision stand-in for the parts of NVIDIA Warp that MPMWarpYDW's
kernels use (TEST INFRASTRUCTURE: used only by gen_golden.py to execute the
reference's own kernel and orchestration source on the CPU).

Warp is not installable here, so this module restates the documented
semantics of the Warp API the reference calls, in numpy float64:

  * ``@wp.kernel`` functions run once per thread index under ``wp.launch``
    (``wp.tid()`` returns the current index; a tuple for a multi-dimensional
    launch), sequentially in index order;
  * ``wp.vec3`` / ``wp.mat33`` are value types: ``mat * mat`` is the matrix
    product, ``mat * vec`` the matrix-vector product, ``mat33(v0, v1, v2)``
    takes the vectors as columns, ``m[i, j]`` indexes, ``m[i]`` is row i;
  * ``wp.svd3(A, U, sigma, V)`` writes A = U diag(sigma) V^T with U, V proper
    rotations and sigma in decreasing order, the last one negative when
    det A < 0;
  * ``wp.normalize`` of a zero vector is zero; ``wp.int`` truncates toward zero;
  * ``wp.HashGrid(dx, dy, dz)``: ``build(points, w)`` puts point p in hash
    ((cz mod dz) * dy + (cy mod dy)) * dx + (cx mod dx), c = max(0, trunc(p/w) + 2^20)
    per axis, and orders points by a stable sort on that hash;
    ``hash_grid_query(grid, x, r)`` visits the cells trunc((x - r)/w) ..
    trunc((x + r)/w) per axis (at most dims cells), x fastest, then y, then z,
    and the points of each cell in sorted order.  Kernels iterate a query with
    ``while wp.hash_grid_query_next(query, index):``; the kernel decorator
    rewrites that loop into a Python ``for index in ...`` over the same order.

Arithmetic is float64 throughout: the kernels execute as written, without
FP32 rounding, which makes the result the precision reference.
"""
from __future__ import annotations

import ast
import inspect
import itertools
import math
import textwrap
import types

import numpy as np

F64 = np.float64

# ---------------------------------------------------------------------------
# scalar types and casts
# ---------------------------------------------------------------------------


def _int(x):
    return int(x)  # truncation toward zero


def _float(x):
    return float(x)


int32 = _int
uint64 = _int
float32 = _float
float64 = _float


# ---------------------------------------------------------------------------
# vec3 / mat33 value types
# ---------------------------------------------------------------------------
class vec3:
    __slots__ = ("a",)
    _len = 3

    def __init__(self, *args):
        if len(args) == 0:
            self.a = np.zeros(3, F64)
        elif len(args) == 1:
            x = args[0]
            if isinstance(x, vec3):
                self.a = x.a.copy()
            elif np.ndim(x) == 0:
                self.a = np.full(3, float(x), F64)
            else:
                self.a = np.array(x, F64).reshape(3)
        elif len(args) == 3:
            self.a = np.array([float(v) for v in args], F64)
        else:
            raise TypeError("vec3 takes 0, 1 or 3 arguments")

    def __getitem__(self, i):
        return float(self.a[i])

    def __setitem__(self, i, v):
        self.a[i] = float(v)

    def __add__(self, o):
        return vec3(self.a + _vec(o))

    def __radd__(self, o):
        return vec3(_vec(o) + self.a)

    def __sub__(self, o):
        return vec3(self.a - _vec(o))

    def __rsub__(self, o):
        return vec3(_vec(o) - self.a)

    def __neg__(self):
        return vec3(-self.a)

    def __mul__(self, o):
        if isinstance(o, mat33):
            return vec3(self.a @ o.a)
        if isinstance(o, vec3):
            raise TypeError("vec3 * vec3 is not defined (use cw_mul or dot)")
        return vec3(self.a * float(o))

    def __rmul__(self, o):
        return vec3(float(o) * self.a)

    def __truediv__(self, o):
        return vec3(self.a / float(o))

    def __repr__(self):
        return f"vec3({self.a[0]}, {self.a[1]}, {self.a[2]})"


def _vec(o):
    if isinstance(o, vec3):
        return o.a
    raise TypeError(f"expected vec3, got {type(o).__name__}")


class mat33:
    __slots__ = ("a",)

    def __init__(self, *args):
        if len(args) == 0:
            self.a = np.zeros((3, 3), F64)
        elif len(args) == 1 and isinstance(args[0], mat33):
            self.a = args[0].a.copy()
        elif len(args) == 1 and np.ndim(args[0]) == 0:
            self.a = np.full((3, 3), float(args[0]), F64)
        elif len(args) == 1:
            self.a = np.array(args[0], F64).reshape(3, 3)
        elif len(args) == 3 and all(isinstance(v, vec3) for v in args):
            self.a = np.stack([v.a for v in args], axis=1)  # columns
        elif len(args) == 9:
            self.a = np.array([float(v) for v in args], F64).reshape(3, 3)
        else:
            raise TypeError("mat33 takes 0, 1, 3 vectors or 9 scalars")

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            return float(self.a[idx])
        return vec3(self.a[idx])

    def __setitem__(self, idx, v):
        if isinstance(idx, tuple):
            self.a[idx] = float(v)
        else:
            self.a[idx] = _vec(v)

    def __add__(self, o):
        return mat33(self.a + o.a)

    def __sub__(self, o):
        return mat33(self.a - o.a)

    def __neg__(self):
        return mat33(-self.a)

    def __mul__(self, o):
        if isinstance(o, mat33):
            return mat33(self.a @ o.a)
        if isinstance(o, vec3):
            return vec3(self.a @ o.a)
        return mat33(self.a * float(o))

    def __rmul__(self, o):
        return mat33(float(o) * self.a)

    def __truediv__(self, o):
        return mat33(self.a / float(o))


# ---------------------------------------------------------------------------
# builtins
# ---------------------------------------------------------------------------
def length(v):
    return float(np.sqrt(np.dot(v.a, v.a)))


def normalize(v):
    n = length(v)
    return vec3(v.a / n) if n > 0.0 else vec3()


def dot(a, b):
    return float(np.dot(a.a, b.a))


def cross(a, b):
    return vec3(np.cross(a.a, b.a))


def outer(a, b):
    return mat33(np.outer(a.a, b.a))


def cw_mul(a, b):
    return vec3(a.a * b.a)


def transpose(m):
    return mat33(m.a.T)


def determinant(m):
    return float(np.linalg.det(m.a))


def ddot(a, b):
    return float(np.sum(a.a * b.a))


def add(a, b):
    return a + b


def sub(a, b):
    return a - b


def _elementwise(fa, fb):
    def f(a, b):
        if isinstance(a, vec3):
            return vec3(fa(a.a, b.a))
        return fb(a, b)
    return f


max = _elementwise(np.maximum, lambda a, b: a if a > b else b)  # noqa: A001
min = _elementwise(np.minimum, lambda a, b: a if a < b else b)  # noqa: A001


def abs(x):  # noqa: A001
    return vec3(np.abs(x.a)) if isinstance(x, vec3) else math.fabs(x)


def sqrt(x):
    return math.sqrt(x)


def log(x):
    return math.log(x)


def exp(x):
    return math.exp(x)


def pow(x, y):  # noqa: A001
    return math.pow(x, y)


def sign(x):
    return -1.0 if x < 0.0 else 1.0


def isnan(x):
    return bool(np.isnan(x.a).any()) if isinstance(x, vec3) else math.isnan(x)


def svd3(A, U, sigma, V):
    """A = U diag(sigma) V^T, U and V rotations, sigma decreasing (last < 0 if det A < 0)."""
    u, s, vt = np.linalg.svd(A.a)
    v = vt.T
    if np.linalg.det(u) < 0:
        u[:, 2] = -u[:, 2]
        s[2] = -s[2]
    if np.linalg.det(v) < 0:
        v[:, 2] = -v[:, 2]
        s[2] = -s[2]
    U.a[...] = u
    sigma.a[...] = s
    V.a[...] = v


# ---------------------------------------------------------------------------
# arrays
# ---------------------------------------------------------------------------
def _inner(dtype):
    if dtype is vec3:
        return (3,)
    if dtype is mat33:
        return (3, 3)
    return ()


def _np_dtype(dtype):
    if dtype in (int, int32, uint64, _int):
        return np.int64
    return F64


class array:
    def __init__(self, data=None, dtype=float, shape=None, device=None, **_):
        self.dtype = dtype
        if data is None and shape is None:
            self.data = None  # an annotation (wp.array(dtype=...))
            return
        if data is not None:
            self.data = np.array(data, dtype=_np_dtype(dtype))
            inner = _inner(dtype)
            if inner and self.data.shape[-len(inner):] != inner:
                self.data = self.data.reshape((-1,) + inner)
        else:
            shp = (shape,) if np.ndim(shape) == 0 else tuple(shape)
            self.data = np.zeros(shp + _inner(dtype), dtype=_np_dtype(dtype))

    @property
    def shape(self):
        return self.data.shape[: self.data.ndim - len(_inner(self.dtype))]

    def _wrap(self, x):
        if self.dtype is vec3:
            return vec3(x)
        if self.dtype is mat33:
            return mat33(x)
        return x.item() if hasattr(x, "item") else x

    def __getitem__(self, idx):
        return self._wrap(self.data[idx])

    def __setitem__(self, idx, v):
        if isinstance(v, (vec3, mat33)):
            self.data[idx] = v.a
        else:
            self.data[idx] = v

    def zero_(self):
        self.data[...] = 0

    def fill_(self, v):
        self.data[...] = np.asarray(v, dtype=self.data.dtype)

    def numpy(self):
        return self.data

    def assign(self, src):
        self.data[...] = src.data if isinstance(src, array) else np.asarray(src)

    def __len__(self):
        return self.data.shape[0]


def zeros(shape=None, dtype=float, device=None, **_):
    return array(shape=shape, dtype=dtype, device=device)


def from_numpy(a, dtype=float, device=None, **_):
    return array(a, dtype=dtype, device=device)


def copy(dest, src, *_, **__):
    dest.data[...] = src.data


def synchronize():
    pass


def init():
    pass


# ---------------------------------------------------------------------------
# kernels and launches
# ---------------------------------------------------------------------------
_TID = [0]


def tid():
    return _TID[0]


class _QueryLoops(ast.NodeTransformer):
    """while wp.hash_grid_query_next(q, name): body  ->  for name in wp._query_points(q): body"""

    def visit_While(self, node):
        self.generic_visit(node)
        t = node.test
        if (isinstance(t, ast.Call) and isinstance(t.func, ast.Attribute) and t.func.attr == "hash_grid_query_next"
                and len(t.args) == 2 and isinstance(t.args[1], ast.Name)):
            it = ast.Call(func=ast.Attribute(value=t.func.value, attr="_query_points", ctx=ast.Load()),
                          args=[t.args[0]], keywords=[])
            return ast.copy_location(ast.For(target=ast.Name(id=t.args[1].id, ctx=ast.Store()), iter=it,
                                             body=node.body, orelse=node.orelse), node)
        return node


def _compile(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    tree = ast.fix_missing_locations(_QueryLoops().visit(tree))
    ns = {}
    exec(compile(tree, inspect.getsourcefile(fn), "exec"), fn.__globals__, ns)
    return ns[fdef.name]


class Kernel:
    def __init__(self, fn):
        self.fn = _compile(fn)
        self.__name__ = fn.__name__


def kernel(fn=None, **_):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def func(fn=None, **_):
    if fn is None:
        return lambda f: _compile(f)
    return _compile(fn)


def launch(kernel, dim, inputs=(), outputs=(), device=None, **_):
    args = list(inputs) + list(outputs)
    if np.ndim(dim) == 0:
        it = range(int(dim))
    else:
        it = itertools.product(*[range(int(d)) for d in dim])
    for t in it:
        _TID[0] = t
        kernel.fn(*args)


def atomic_add(arr, *rest):
    *idx, value = rest
    idx = tuple(int(i) for i in idx)
    if isinstance(value, (vec3, mat33)):
        arr.data[idx] += value.a
    else:
        arr.data[idx] += value


# ---------------------------------------------------------------------------
# hash grid
# ---------------------------------------------------------------------------
class HashGrid:
    def __init__(self, dim_x, dim_y, dim_z, device=None):
        self.dims = (int(dim_x), int(dim_y), int(dim_z))
        self.id = self
        self.cell_width = 1.0
        self.point_ids = np.zeros(0, np.int64)
        self.cell_starts = {}
        self.cell_ends = {}

    def _hash(self, cx, cy, cz):
        o = 1 << 20
        c = [max(0, cx + o), max(0, cy + o), max(0, cz + o)]
        dx, dy, dz = self.dims
        return ((c[2] % dz) * dy + (c[1] % dy)) * dx + (c[0] % dx)

    def build(self, points, radius):
        w = float(radius)
        self.cell_width = w
        inv = 1.0 / w
        p = points.data
        keys = np.array([self._hash(int(p[i, 0] * inv), int(p[i, 1] * inv), int(p[i, 2] * inv))
                         for i in range(p.shape[0])], np.int64)
        order = np.argsort(keys, kind="stable")
        self.point_ids = order
        sk = keys[order]
        self.cell_starts, self.cell_ends = {}, {}
        for i, k in enumerate(sk):
            k = int(k)
            if k not in self.cell_starts:
                self.cell_starts[k] = i
            self.cell_ends[k] = i + 1


class _Query:
    def __init__(self, grid, x, r):
        self.grid, self.x, self.r = grid, x, float(r)


def hash_grid_point_id(grid, i):
    return int(grid.point_ids[int(i)])


def hash_grid_query(grid, x, r):
    return _Query(grid, x, r)


def _query_points(q):
    g = q.grid
    inv = 1.0 / g.cell_width
    lo = [int((q.x[a] - q.r) * inv) for a in range(3)]
    hi = [int((q.x[a] + q.r) * inv) for a in range(3)]
    hi = [builtin_min(hi[a], lo[a] + g.dims[a] - 1) for a in range(3)]
    for cz in range(lo[2], hi[2] + 1):
        for cy in range(lo[1], hi[1] + 1):
            for cx in range(lo[0], hi[0] + 1):
                h = g._hash(cx, cy, cz)
                for s in range(g.cell_starts.get(h, 0), g.cell_ends.get(h, 0)):
                    yield int(g.point_ids[s])


builtin_min = __builtins__["min"] if isinstance(__builtins__, dict) else __builtins__.min

# the kernels reach these through the module object
float = float  # noqa: A001,PLW0127  (wp.float in annotations and casts)
int = int  # noqa: A001,PLW0127


def install():
    """Register this module as ``warp`` (sys.modules) and return it."""
    import sys
    mod = sys.modules[__name__]
    sys.modules["warp"] = mod
    return mod


_ = types
