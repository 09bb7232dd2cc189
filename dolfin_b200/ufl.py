"""A small form language with UFL's spelling, and the recogniser that maps a
form to one of the engine's element kernels.

There is no form compiler in the engine (DOLFIN hands UFL forms to FFC,
python/dolfin/fem/form.py:43-53, python/dolfin/jit/jit.py:91-97).  Instead,
an integrand built from TestFunction/TrialFunction, Function, Constant and
the operators below is evaluated numerically on random probe values of the
arguments' values and gradients, and identified as one of the named forms:

    kappa * inner(grad(u), grad(v)) * dx     kappa: 1, Constant, P1 Function, c*Function
    inner(sigma(u), epsilon(v)) * dx          2 mu eps:eps + lmbda div div  (mu, lmbda fitted)
    f * v * dx, inner(f, v) * dx             f: Constant (vector), P1 Function, c*Function
    w * u * v * ds                            boundary mass (Robin), w as kappa (scalar spaces)
    g * v * ds, inner(t, v) * ds              Neumann load, g as f; t a constant vector
    w * dx, w * ds                            functionals: w = Constant, P1 Function, c*x[i]

A form may hold dx and ds terms (cell part + exterior-facet part, assembled
as the reference's cell loop followed by its exterior-facet loop).  Anything
else raises NotImplementedError: no other kernels exist.
"""
from __future__ import annotations

import numbers

import numpy as np

_NPROBE = 7


class Expr:
    shape = ()

    # -- algebra -----------------------------------------------------------
    def __add__(self, o):
        return Sum(self, as_expr(o))

    __radd__ = __add__

    def __sub__(self, o):
        return Sum(self, Product(ScalarValue(-1.0), as_expr(o)))

    def __rsub__(self, o):
        return Sum(as_expr(o), Product(ScalarValue(-1.0), self))

    def __neg__(self):
        return Product(ScalarValue(-1.0), self)

    def __mul__(self, o):
        if isinstance(o, Measure):
            return Form([(self, o)])
        return Product(self, as_expr(o))

    def __rmul__(self, o):
        return Product(as_expr(o), self)

    def __truediv__(self, o):
        return Product(self, ScalarValue(1.0 / float(o)))

    @property
    def T(self):
        return Transpose(self)

    def __getitem__(self, i):
        return Indexed(self, i)

    def ev(self, env):  # -> ndarray (NPROBE, *shape)
        raise NotImplementedError

    def walk(self):
        yield self
        for c in getattr(self, "ops", ()):
            yield from c.walk()


def as_expr(o):
    if isinstance(o, Expr):
        return o
    if isinstance(o, numbers.Number):
        return ScalarValue(float(o))
    raise TypeError(f"cannot use {type(o).__name__} in a form")


class ScalarValue(Expr):
    def __init__(self, v):
        self.v = float(v)
        self.ops = ()

    def ev(self, env):
        return np.full((_NPROBE,), self.v)


class Argument(Expr):
    def __init__(self, V, number):
        self.V, self.number, self.ops = V, number, ()
        vs = V.value_size()
        self.shape = () if vs == 1 else (vs,)

    def ev(self, env):
        return env["val"][self.number]


def TestFunction(V):
    return Argument(V, 0)


def TrialFunction(V):
    return Argument(V, 1)


class Identity(Expr):
    def __init__(self, d):
        self.d, self.ops = d, ()
        self.shape = (d, d)

    def ev(self, env):
        return np.broadcast_to(np.eye(self.d), (_NPROBE, self.d, self.d)).copy()


class Grad(Expr):
    def __init__(self, f):
        f = as_expr(f)
        if not isinstance(f, Argument):
            raise NotImplementedError("grad() is provided for test/trial functions only")
        self.ops = (f,)
        d = f.V.mesh().geometry_dim()
        self.shape = f.shape + (d,)

    def ev(self, env):
        return env["grad"][self.ops[0].number]


def grad(f):
    return Grad(f)


def nabla_grad(f):
    return Transpose(Grad(f)) if as_expr(f).shape else Grad(f)


class Transpose(Expr):
    def __init__(self, A):
        self.ops = (as_expr(A),)
        s = self.ops[0].shape
        if len(s) != 2:
            raise ValueError("transpose of a non-matrix")
        self.shape = (s[1], s[0])

    def ev(self, env):
        return np.swapaxes(self.ops[0].ev(env), 1, 2)


def transpose(A):
    return Transpose(A)


class Sum(Expr):
    def __init__(self, a, b):
        a, b = as_expr(a), as_expr(b)
        if a.shape != b.shape:
            raise ValueError(f"shape mismatch in sum: {a.shape} vs {b.shape}")
        self.ops, self.shape = (a, b), a.shape

    def ev(self, env):
        return self.ops[0].ev(env) + self.ops[1].ev(env)


class Product(Expr):
    def __init__(self, a, b):
        a, b = as_expr(a), as_expr(b)
        if a.shape and b.shape:
            raise ValueError("product of two non-scalars: use inner/dot")
        self.ops, self.shape = (a, b), a.shape or b.shape

    def ev(self, env):
        x, y = self.ops[0].ev(env), self.ops[1].ev(env)
        if x.ndim < y.ndim:
            x = x.reshape(x.shape + (1,) * (y.ndim - x.ndim))
        elif y.ndim < x.ndim:
            y = y.reshape(y.shape + (1,) * (x.ndim - y.ndim))
        return x * y


class Inner(Expr):
    def __init__(self, a, b):
        a, b = as_expr(a), as_expr(b)
        if a.shape != b.shape:
            raise ValueError(f"inner: shapes {a.shape} and {b.shape} differ")
        self.ops = (a, b)

    def ev(self, env):
        p = self.ops[0].ev(env) * self.ops[1].ev(env)
        return p.reshape(_NPROBE, -1).sum(axis=1)


def inner(a, b):
    return Inner(a, b)


class Dot(Expr):
    def __init__(self, a, b):
        a, b = as_expr(a), as_expr(b)
        if not a.shape or not b.shape or a.shape[-1] != b.shape[0]:
            raise ValueError("dot: incompatible shapes")
        self.ops = (a, b)
        self.shape = a.shape[:-1] + b.shape[1:]

    def ev(self, env):
        x, y = self.ops[0].ev(env), self.ops[1].ev(env)
        return np.einsum("p...i,pi...->p...", x, y)


def dot(a, b):
    a, b = as_expr(a), as_expr(b)
    if not a.shape and not b.shape:
        return Product(a, b)
    return Dot(a, b)


class Trace(Expr):
    def __init__(self, A):
        self.ops = (as_expr(A),)

    def ev(self, env):
        return np.trace(self.ops[0].ev(env), axis1=1, axis2=2)


def tr(A):
    return Trace(A)


def sym(A):
    return 0.5 * (A + Transpose(A))


def div(f):
    f = as_expr(f)
    if not f.shape:
        raise ValueError("div of a scalar")
    return Trace(Grad(f))


class Indexed(Expr):
    def __init__(self, f, i):
        self.ops, self.i = (as_expr(f),), i
        self.shape = self.ops[0].shape[1:]

    def ev(self, env):
        return self.ops[0].ev(env)[:, self.i]


class SpatialCoordinate(Expr):
    """x = SpatialCoordinate(mesh); x[i] is the i-th coordinate (P1 on affine cells)."""

    def __init__(self, mesh):
        self.mesh, self.ops = mesh, ()
        self.shape = (mesh.geometry_dim(),)

    def ev(self, env):
        return env["x"]


class Measure:
    """dx (cells) or ds (exterior facets), optionally bound to a mesh: dx(mesh)."""

    def __init__(self, name="dx", domain=None):
        self.name, self.domain = name, domain

    def __call__(self, *a, domain=None, subdomain_data=None, subdomain_id=None, **k):
        if a and hasattr(a[0], "geometry_dim"):
            domain, a = a[0], a[1:]
        if a or k or subdomain_data is not None or subdomain_id is not None:
            raise NotImplementedError("subdomain integrals are not provided")
        return Measure(self.name, domain if domain is not None else self.domain)

    def __rmul__(self, integrand):
        return Form([(as_expr(integrand), self)])


dx = Measure("dx")
ds = Measure("ds")


class Form:
    def __init__(self, terms):
        for _, m in terms:
            if m.name not in ("dx", "ds"):
                raise NotImplementedError(
                    f"cell (dx) and exterior facet (ds) integrals are provided, got {m.name}")
        self.terms = list(terms)

    def part(self, name):
        """The terms integrated over measure `name` ("dx" or "ds"), or None."""
        t = [(e, m) for e, m in self.terms if m.name == name]
        return Form(t) if t else None

    def measures(self):
        return sorted({m.name for _, m in self.terms})

    def domain(self):
        """The mesh of the form: from its measures, arguments or coefficients."""
        for _, m in self.terms:
            if m.domain is not None:
                return m.domain
        for n in self.integrand().walk():
            if isinstance(n, Argument):
                return n.V.mesh()
            if isinstance(n, SpatialCoordinate):
                return n.mesh
            if hasattr(n, "function_space"):
                return n.function_space().mesh()
        return None

    def __add__(self, o):
        return Form(self.terms + o.terms)

    def __sub__(self, o):
        return Form(self.terms + [(Product(ScalarValue(-1.0), e), m) for e, m in o.terms])

    def __neg__(self):
        return Form([(Product(ScalarValue(-1.0), e), m) for e, m in self.terms])

    def __rmul__(self, c):
        return Form([(Product(as_expr(c), e), m) for e, m in self.terms])

    def integrand(self):
        e = self.terms[0][0]
        for t, _ in self.terms[1:]:
            e = Sum(e, t)
        return e

    def arguments(self):
        args = {}
        for n in self.integrand().walk():
            if isinstance(n, Argument):
                if n.number in args and args[n.number] is not n.V:
                    raise ValueError("argument defined on two spaces")
                args[n.number] = n.V
        return args

    def coefficients(self):
        from .function import Constant, Function
        fs, cs = [], []
        for n in self.integrand().walk():
            if isinstance(n, Function) and n not in fs:
                fs.append(n)
            if isinstance(n, Constant) and n not in cs:
                cs.append(n)
        return fs, cs

    def rank(self):
        return len(self.arguments())


# ---------------------------------------------------------------------------
# Recogniser
# ---------------------------------------------------------------------------
class Recognised:
    """Identified form: kind, coefficient, constants, space."""

    def __init__(self, kind, V, coeff, function=None, constant=(0.0, 0.0, 0.0), mu=0.0, lmbda=0.0,
                 pair=None):
        self.kind, self.V, self.coeff = kind, V, coeff
        self.function, self.constant, self.mu, self.lmbda = function, tuple(constant), mu, lmbda
        # a load c*f1*f2*v*dx: the two P1 Functions (which one is kappa is
        # decided by the bilinear form it is assembled with)
        self.pair = pair

    def with_kappa(self, kappa):
        """The load c*kappa*f*v*dx of a two-Function load, kappa being the
        bilinear form's coefficient: DB2_COEFF_P1_KAPPA with f."""
        from . import _capi
        if self.pair is None or kappa is None or not any(kappa is g for g in self.pair):
            raise NotImplementedError("a load with two Functions is provided as kappa*f*v*dx, kappa "
                                      "being the bilinear form's coefficient (SystemAssembler)")
        f = self.pair[1] if self.pair[0] is kappa else self.pair[0]
        return Recognised(self.kind, self.V, _capi.COEFF_P1_KAPPA, f, self.constant)

    def c_form(self):
        from . import _capi
        return _capi.make_form(self.kind, self.coeff, self.constant, self.mu, self.lmbda)

    def __repr__(self):
        return (f"Recognised(kind={self.kind}, coeff={self.coeff}, constant={self.constant}, "
                f"mu={self.mu}, lmbda={self.lmbda})")


def _env(rng, args, fvals=None, zero_values=False, zero_grads=False):
    env = {"val": {}, "grad": {}, "f": fvals or {}}
    for V in args.values():
        env["x"] = rng.standard_normal((_NPROBE, V.mesh().geometry_dim()))
    for num, V in args.items():
        vs, d = V.value_size(), V.mesh().geometry_dim()
        vshape = (_NPROBE,) if vs == 1 else (_NPROBE, vs)
        gshape = (_NPROBE, d) if vs == 1 else (_NPROBE, vs, d)
        env["val"][num] = np.zeros(vshape) if zero_values else rng.standard_normal(vshape)
        env["grad"][num] = np.zeros(gshape) if zero_grads else rng.standard_normal(gshape)
    return env


def _close(a, b, tol=1e-10):
    return np.allclose(a, b, rtol=tol, atol=tol * (1.0 + np.max(np.abs(b))))


def recognise_parts(form):
    """(cell part, exterior-facet part) of a rank 1/2 form, each a Recognised
    or None."""
    if not isinstance(form, Form):
        raise TypeError("expected a Form")
    fx, fs = form.part("dx"), form.part("ds")
    cell = recognise(fx) if fx is not None else None
    facet = recognise_facet(fs) if fs is not None else None
    if cell is not None and facet is not None and cell.V is not facet.V:
        raise ValueError("dx and ds terms on different spaces")
    return cell, facet


def recognise_facet(form):
    """Exterior-facet part: w*u*v*ds, g*v*ds or inner(t, v)*ds."""
    from . import _capi
    args = form.arguments()
    rank = len(args)
    fs, _ = form.coefficients()
    if len(fs) > 1:
        raise NotImplementedError("ds forms with more than one Function coefficient are not provided")
    func = fs[0] if fs else None
    if func is not None and (func.function_space().degree() != 1 or func.function_space().value_size() != 1):
        raise NotImplementedError("coefficients must be scalar P1 Functions")
    rng = np.random.default_rng(20190402)
    I = form.integrand()

    def ev(env):
        return I.ev(env)

    def fvals(v):
        return {func: np.full(_NPROBE, v)} if func is not None else {}

    if rank == 2:
        V = args[0]
        if args[1] is not V:
            raise NotImplementedError("rectangular (V x W) forms are not provided")
        if V.value_size() != 1:
            raise NotImplementedError("boundary mass on vector spaces is not provided")
        env = _env(rng, args, fvals(1.0))
        full = ev(env)
        env0 = dict(env, grad={k: np.zeros_like(v) for k, v in env["grad"].items()})
        if not _close(ev(env0), full):
            raise NotImplementedError("only w*u*v*ds bilinear facet forms are provided")
        uv = env["val"][0] * env["val"][1]
        A1 = full / uv
        if not np.allclose(A1, A1[0], rtol=1e-10):
            raise NotImplementedError("bilinear facet form is not w*u*v*ds")
        alpha = _unit_probe(ev, args, fvals(1.0), grads=False)
        if func is None:
            coeff = _capi.COEFF_NONE if alpha == 1.0 else _capi.COEFF_CONSTANT
            return Recognised(_capi.FORM_FACET_MASS, V, coeff, None, (alpha, 0, 0))
        A2 = ev(dict(env, f=fvals(2.0))) / uv
        if not _close(A2, 2.0 * A1):
            raise NotImplementedError("coefficient must enter linearly as a factor")
        coeff = _capi.COEFF_P1 if alpha == 1.0 else _capi.COEFF_P1_SCALED
        return Recognised(_capi.FORM_FACET_MASS, V, coeff, func, (alpha, 0, 0))
    if rank == 1:
        # the linear recogniser, with the facet kind
        r = recognise(form, _kind=_capi.FORM_FACET_LOAD)
        return r
    raise NotImplementedError("use assemble() for functionals")


def recognise_functional(form):
    """Rank-0 form: [(kind, mesh, coeff, function, constant)] for its dx / ds
    parts; integrands c, c*f (P1 Function f) or c*x[i]."""
    from . import _capi
    from .function import Function
    if form.rank() != 0:
        raise ValueError("not a functional")
    out = []
    for name, kind in (("dx", _capi.FORM_FUNCTIONAL), ("ds", _capi.FORM_FACET_FUNCTIONAL)):
        part = form.part(name)
        if part is None:
            continue
        mesh = part.domain() or form.domain()
        if mesh is None:
            raise ValueError("functional without a mesh: integrate over dx(mesh) / ds(mesh)")
        I = part.integrand()
        fs = [n for n in I.walk() if isinstance(n, Function)]
        xs = [n for n in I.walk() if isinstance(n, SpatialCoordinate)]
        if len(set(map(id, fs))) > 1 or (fs and xs):
            raise NotImplementedError("functionals of one P1 Function or one coordinate are provided")
        rng = np.random.default_rng(20190403)
        gd = mesh.geometry_dim()
        env = {"val": {}, "grad": {}, "f": {}, "x": rng.standard_normal((_NPROBE, gd))}
        if fs:
            f = fs[0]
            if f.function_space().degree() != 1 or f.function_space().value_size() != 1:
                raise NotImplementedError("functional coefficients must be scalar P1 Functions")
            v1 = I.ev(dict(env, f={f: np.ones(_NPROBE)}))
            v2 = I.ev(dict(env, f={f: np.full(_NPROBE, 2.0)}))
            if not (np.allclose(v1, v1[0], rtol=1e-12) and _close(v2, 2.0 * v1)):
                raise NotImplementedError("functional must be c * f for a P1 Function f")
            alpha = float(v1[0])
            coeff = _capi.COEFF_P1 if alpha == 1.0 else _capi.COEFF_P1_SCALED
            out.append((kind, mesh, coeff, f, (alpha, 0.0, 0.0)))
        elif xs:
            full = I.ev(env)
            alphas = []
            for i in range(gd):
                e = np.zeros((_NPROBE, gd))
                e[:, i] = 1.0
                alphas.append(float(I.ev(dict(env, x=e))[0]))
            if not _close(env["x"] @ np.array(alphas), full) or sum(a != 0.0 for a in alphas) != 1:
                raise NotImplementedError("functional must be c * x[i]")
            i = next(k for k, a in enumerate(alphas) if a != 0.0)
            out.append((kind, mesh, _capi.COEFF_COORD, None, (alphas[i], float(i), 0.0)))
        else:
            v = I.ev(env)
            if not np.allclose(v, v[0], rtol=1e-12):
                raise NotImplementedError("functional integrand is not constant")
            out.append((kind, mesh, _capi.COEFF_CONSTANT, None, (float(v[0]), 0.0, 0.0)))
    return out


def recognise(form, _kind=None):
    """Cell (dx) part of a rank 1/2 form: one of the engine's cell kernels."""
    from . import _capi
    if not isinstance(form, Form):
        raise TypeError("expected a Form")
    if _kind is None and "ds" in form.measures():
        if "dx" not in form.measures():
            raise NotImplementedError("the form has only ds terms: use recognise_parts")
        form = form.part("dx")
    args = form.arguments()
    rank = len(args)
    fs, _ = form.coefficients()
    if len(fs) == 2 and rank == 1 and _kind is None:
        return _recognise_pair_load(form, args, fs)
    if len(fs) > 1:
        raise NotImplementedError("forms with more than one Function coefficient are not provided")
    func = fs[0] if fs else None
    if func is not None and (func.function_space().degree() != 1 or func.function_space().value_size() != 1):
        raise NotImplementedError("coefficients must be scalar P1 Functions")
    rng = np.random.default_rng(20190401)
    I = form.integrand()

    def ev(env):
        return I.ev(env)

    def fvals(v):
        return {func: np.full(_NPROBE, v)} if func is not None else {}

    if rank == 2:
        V0, V1 = args[0], args[1]
        if V0 is not V1:
            raise NotImplementedError("rectangular (V x W) forms are not provided")
        V = V0
        if V.mesh() is not (func.function_space().mesh() if func else V.mesh()):
            raise ValueError("coefficient lives on another mesh")
        env = _env(rng, args, fvals(1.0))
        full = ev(env)
        envg = dict(env, val={k: np.zeros_like(v) for k, v in env["val"].items()})
        if not _close(ev(envg), full):
            raise NotImplementedError("only gradient-gradient bilinear forms are provided (no mass terms)")
        if V.value_size() == 1:
            g = np.einsum("pi,pi->p", env["grad"][0], env["grad"][1])
            K1 = full / g
            if not np.allclose(K1, K1[0], rtol=1e-10):
                raise NotImplementedError("bilinear form is not kappa*inner(grad(u), grad(v))")
            alpha = _unit_probe(ev, args, fvals(1.0), grads=True)
            if func is None:
                coeff = _capi.COEFF_NONE if alpha == 1.0 else _capi.COEFF_CONSTANT
                return Recognised(_capi.FORM_DIFFUSION, V, coeff, None, (alpha, 0, 0))
            env2 = dict(env, f=fvals(2.0))
            K2 = ev(env2) / g
            if not _close(K2, 2.0 * K1):
                raise NotImplementedError("coefficient must enter linearly as a factor")
            coeff = _capi.COEFF_P1 if alpha == 1.0 else _capi.COEFF_P1_SCALED
            return Recognised(_capi.FORM_DIFFUSION, V, coeff, func, (alpha, 0, 0))
        # vector: fit 2 mu eps(u):eps(v) + lmbda div(u) div(v)
        if func is not None:
            raise NotImplementedError("elasticity with a Function coefficient is not provided")
        Gu, Gv = env["grad"][1], env["grad"][0]
        epsu = 0.5 * (Gu + np.swapaxes(Gu, 1, 2))
        epsv = 0.5 * (Gv + np.swapaxes(Gv, 1, 2))
        b1 = 2.0 * np.einsum("pij,pij->p", epsu, epsv)
        b2 = np.trace(Gu, axis1=1, axis2=2) * np.trace(Gv, axis1=1, axis2=2)
        M = np.stack([b1, b2], axis=1)
        sol, *_ = np.linalg.lstsq(M, full, rcond=None)
        if not _close(M @ sol, full):
            raise NotImplementedError("vector bilinear form is not inner(sigma(u), epsilon(v))")
        mu, lmbda = float(sol[0]), float(sol[1])
        # round-off from the fit: snap to the values the Constants carry
        mu, lmbda = _snap(mu, form), _snap(lmbda, form)
        return Recognised(_capi.FORM_ELASTICITY, V, _capi.COEFF_NONE, None, (0, 0, 0), mu, lmbda)

    if rank == 1:
        lkind = _kind if _kind is not None else _capi.FORM_LOAD
        V = args[0]
        env = _env(rng, args, fvals(1.0))
        full = ev(env)
        env0 = dict(env, grad={k: np.zeros_like(v) for k, v in env["grad"].items()})
        if not _close(ev(env0), full):
            raise NotImplementedError("only f*v*dx / inner(f, v)*dx linear forms are provided")
        if V.value_size() == 1:
            F1 = full / env["val"][0]
            if not np.allclose(F1, F1[0], rtol=1e-10):
                raise NotImplementedError("linear form is not f*v*dx")
            alpha = _unit_probe(ev, args, fvals(1.0), grads=False)
            if func is None:
                return Recognised(lkind, V, _capi.COEFF_CONSTANT, None, (alpha, 0, 0))
            F2 = ev(dict(env, f=fvals(2.0))) / env["val"][0]
            if not _close(F2, 2.0 * F1):
                raise NotImplementedError("load coefficient must enter linearly")
            coeff = _capi.COEFF_P1 if alpha == 1.0 else _capi.COEFF_P1_SCALED
            return Recognised(lkind, V, coeff, func, (alpha, 0, 0))
        if func is not None:
            raise NotImplementedError("vector loads take a Constant")
        vs = V.value_size()
        fvec = []
        for c in range(vs):
            e = dict(env, val={0: np.tile(np.eye(vs)[c], (_NPROBE, 1))})
            fvec.append(float(ev(e)[0]))
        chk = np.einsum("pi,i->p", env["val"][0], np.array(fvec))
        if not _close(chk, full):
            raise NotImplementedError("vector load is not inner(f, v) with constant f")
        return Recognised(lkind, V, _capi.COEFF_CONSTANT, None, tuple(fvec) + (0.0,) * (3 - vs))

    raise NotImplementedError("functionals: use assemble() (rank-0 forms)")


def _recognise_pair_load(form, args, fs):
    """c*f1*f2*v*dx with two scalar P1 Functions (the kappa-weighted load
    kappa*f*v*dx of an adjoint problem)."""
    from . import _capi
    for g in fs:
        if g.function_space().degree() != 1 or g.function_space().value_size() != 1:
            raise NotImplementedError("coefficients must be scalar P1 Functions")
    V = args[0]
    if V.value_size() != 1:
        raise NotImplementedError("a load with two Functions is provided on scalar spaces")
    rng = np.random.default_rng(20190404)
    I = form.integrand()
    f1, f2 = fs

    def fv(a, b):
        return {f1: np.full(_NPROBE, a), f2: np.full(_NPROBE, b)}

    env = _env(rng, args, fv(1.0, 1.0))
    full = I.ev(env)
    env0 = dict(env, grad={k: np.zeros_like(v) for k, v in env["grad"].items()})
    if not _close(I.ev(env0), full):
        raise NotImplementedError("only c*f*g*v*dx loads with two Functions are provided")
    F1 = full / env["val"][0]
    if not np.allclose(F1, F1[0], rtol=1e-10):
        raise NotImplementedError("linear form is not c*f*g*v*dx")
    for a, b in ((2.0, 1.0), (1.0, 2.0), (3.0, 5.0)):
        if not _close(I.ev(dict(env, f=fv(a, b))) / env["val"][0], a * b * F1):
            raise NotImplementedError("the two Functions must enter as a product factor")
    alpha = _unit_probe(lambda e: I.ev(e), args, fv(1.0, 1.0), grads=False)
    return Recognised(_capi.FORM_LOAD, V, _capi.COEFF_P1_KAPPA, None, (alpha, 0, 0), pair=(f1, f2))


def _unit_probe(ev, args, fv, grads):
    """Integrand at unit arguments (grad u = grad v = e_0, or v = 1) and unit
    coefficient values: the exact scalar factor of a recognised form."""
    env = {"val": {}, "grad": {}, "f": fv}
    for num, V in args.items():
        d = V.mesh().geometry_dim()
        g = np.zeros((_NPROBE, d))
        g[:, 0] = 1.0
        env["val"][num] = np.zeros(_NPROBE) if grads else np.ones(_NPROBE)
        env["grad"][num] = g if grads else np.zeros((_NPROBE, d))
    return float(ev(env)[0])


def _snap(v, form):
    """Replace a least-squares value by the nearest exact combination 0.5*c or c
    of the form's Constants when within 1e-12 (keeps mu, lmbda bit-exact)."""
    _, cs = form.coefficients()
    cands = [0.0]
    for c in cs:
        if c.value_size() == 1:
            x = float(c.values()[0])
            cands += [x, 0.5 * x, 2.0 * x]
    for c in cands:
        if abs(v - c) <= 1e-12 * max(1.0, abs(c)):
            return c
    return v
