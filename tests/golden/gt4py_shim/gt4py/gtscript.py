"""Minimal stand-in for ``gt4py.gtscript`` (gt4py v36) used only to execute the
reference's stencil definitions on the CPU when generating golden fixtures.

This is test infrastructure.  It implements the subset of gtscript that the
acoustic-substep stencils use, with the semantics of gt4py's ``numpy``
backend as the reference relies on them:

* every statement of a ``computation(PARALLEL)`` block is applied over its
  whole (extended) box before the next statement runs;
* ``FORWARD`` / ``BACKWARD`` computations iterate k sequentially, running the
  statements of every interval that contains k;
* temporaries (and API fields that are read with a horizontal offset later in
  the same stencil) are computed over the box that later reads need
  (extent analysis), API fields at least over the call domain;
* ``horizontal(region[...])`` restricts an assignment to absolute index sets
  relative to the call domain; it never enlarges the box;
* ``gtscript.function`` calls are inlined; ``__INLINED`` and externals are
  compile-time constants; field ``if`` statements become masked assignments
  whose condition is evaluated once, before the branch body.
"""
import ast
import inspect
import textwrap

import numpy as np

# ---------------------------------------------------------------- markers
PARALLEL = "PARALLEL"
FORWARD = "FORWARD"
BACKWARD = "BACKWARD"


def computation(order):  # only ever parsed, never executed
    raise RuntimeError("gtscript.computation used outside a stencil")


def interval(*args):
    raise RuntimeError("gtscript.interval used outside a stencil")


def horizontal(*args):
    raise RuntimeError("gtscript.horizontal used outside a stencil")


class _RegionMaker:
    def __getitem__(self, item):
        raise RuntimeError("gtscript.region used outside a stencil")


region = _RegionMaker()


def __INLINED(x):  # noqa: N802
    return x


def compile_assert(x):
    return x


_INLINED_FN = globals()["__INLINED"]


# math functions (only their names matter inside stencils)
exp = np.exp
log = np.log
sqrt = np.sqrt
floor = np.floor
ceil = np.ceil
sin = np.sin
cos = np.cos
tan = np.tan
asin = np.arcsin
acos = np.arccos
atan = np.arctan
isnan = np.isnan

_MATH = {
    "exp": np.exp,
    "log": np.log,
    "sqrt": np.sqrt,
    "floor": np.floor,
    "ceil": np.ceil,
    "sin": np.sin,
    "cos": np.cos,
    "tan": np.tan,
    "asin": np.arcsin,
    "acos": np.arccos,
    "atan": np.arctan,
    "abs": np.abs,
    "isnan": np.isnan,
    "trunc": np.trunc,
}


# ---------------------------------------------------------------- axes
class AxisIndex:
    """An index along I or J relative to the start or end of the call domain."""

    def __init__(self, axis, level, offset):
        self.axis = axis
        self.level = level  # "start" or "end"
        self.offset = int(offset)

    def __add__(self, other):
        return AxisIndex(self.axis, self.level, self.offset + int(other))

    def __radd__(self, other):
        return self.__add__(other)

    def __sub__(self, other):
        return AxisIndex(self.axis, self.level, self.offset - int(other))

    def resolve(self, n):
        return self.offset if self.level == "start" else n + self.offset

    def __repr__(self):
        return f"{self.axis}[{self.level}{self.offset:+d}]"


class _Axis:
    def __init__(self, name):
        self.name = name

    def __getitem__(self, k):
        k = int(k)
        if k >= 0:
            return AxisIndex(self.name, "start", k)
        return AxisIndex(self.name, "end", k)

    def __repr__(self):
        return self.name


I = _Axis("I")  # noqa: E741
J = _Axis("J")
K = _Axis("K")
IJ = "IJ"
IJK = "IJK"
IK = "IK"
JK = "JK"


class FieldDescriptor:
    def __init__(self, axes, dtype):
        if isinstance(axes, _Axis):
            axes = axes.name
        self.axes = str(axes)
        self.dtype = dtype

    def __repr__(self):
        return f"Field[{self.axes}]"


class _FieldMaker:
    def __getitem__(self, item):
        if isinstance(item, tuple):
            axes, dtype = item
        else:
            axes, dtype = IJK, item
        return FieldDescriptor(axes, dtype)


Field = _FieldMaker()


def function(func):
    func.__gtscript_function__ = True
    return func


# ---------------------------------------------------------------- IR
class _Stmt:
    __slots__ = ("target", "expr", "cond", "regions", "comp", "block", "reads", "idx")

    def __init__(self, target, expr, cond, regions, comp, block):
        self.target = target
        self.expr = expr
        self.cond = cond
        self.regions = regions
        self.comp = comp
        self.block = block


class _Loop:
    """A ``while`` loop: ``body`` starts with the statement that evaluates the
    loop test into ``test``; ``active`` is the mask under which the body runs
    (the enclosing condition and the test)."""

    __slots__ = ("body", "active", "comp", "block", "idx")

    def __init__(self, body, active, comp, block):
        self.body = body
        self.active = active
        self.comp = comp
        self.block = block


class _Comp:
    def __init__(self, order):
        self.order = order
        self.blocks = []  # list of (interval (a, b), [stmts])


def _expr_reads(e, out):
    tag = e[0]
    if tag == "f":
        out.append((e[1], e[2][0], e[2][1]))
        if not isinstance(e[2][2], int):
            _expr_reads(e[2][2][1], out)
    elif tag in ("bin", "cmp"):
        _expr_reads(e[2], out)
        _expr_reads(e[3], out)
    elif tag == "un":
        _expr_reads(e[2], out)
    elif tag == "bool":
        for x in e[2]:
            _expr_reads(x, out)
    elif tag == "ifexp":
        _expr_reads(e[1], out)
        _expr_reads(e[2], out)
        _expr_reads(e[3], out)
    elif tag == "call":
        for x in e[2]:
            _expr_reads(x, out)


_BINOPS = {
    ast.Add: "+",
    ast.Sub: "-",
    ast.Mult: "*",
    ast.Div: "/",
    ast.Pow: "**",
    ast.Mod: "%",
    ast.FloorDiv: "//",
}
_CMPOPS = {
    ast.Lt: "<",
    ast.LtE: "<=",
    ast.Gt: ">",
    ast.GtE: ">=",
    ast.Eq: "==",
    ast.NotEq: "!=",
}

_SOURCE_CACHE = {}


def _parse_function(func):
    key = func
    if key not in _SOURCE_CACHE:
        src = textwrap.dedent(inspect.getsource(func))
        tree = ast.parse(src)
        fdef = tree.body[0]
        assert isinstance(fdef, ast.FunctionDef), func
        _SOURCE_CACHE[key] = fdef
    return _SOURCE_CACHE[key]


def _assigned_names(body):
    names = set()
    for node in body:
        for sub in ast.walk(node):
            if isinstance(sub, ast.Assign):
                for t in sub.targets:
                    for n in ast.walk(t):
                        if isinstance(n, ast.Name):
                            names.add(n.id)
            elif isinstance(sub, ast.AugAssign) and isinstance(sub.target, ast.Name):
                names.add(sub.target.id)
    return names


class _Lowering:
    def __init__(self, definition, externals, params):
        self.externals = dict(externals)
        self.params = params  # name -> ("field", axes) | ("scalar", None)
        self.comps = []
        self.temps = {}
        self.n_fresh = 0
        self.cur_comp = None
        self.cur_block = None
        self.definition = definition

    # ---------------- helpers
    def fresh(self, hint="t"):
        self.n_fresh += 1
        name = f"__{hint}{self.n_fresh}"
        self.temps[name] = True
        return name

    def emit(self, target, expr, ctx):
        if self.cur_block is None:
            raise SyntaxError("assignment outside computation/interval")
        st = _Stmt(target, expr, ctx["cond"], ctx["regions"], self.cur_comp, self.cur_block)
        self.cur_block[1].append(st)

    # ---------------- name resolution
    def lookup(self, name, env, globs):
        if name in env:
            return env[name]
        if name in globs:
            return self.classify(globs[name])
        import builtins

        if name in ("abs", "min", "max"):
            return ("math", name)
        if hasattr(builtins, name):
            return ("const", getattr(builtins, name))
        raise NameError(f"gtscript shim: unknown name {name!r}")

    def classify(self, obj):
        if getattr(obj, "__gtscript_function__", False):
            return ("func", obj)
        if inspect.ismodule(obj):
            return ("mod", obj)
        if isinstance(obj, AxisIndex):
            return ("axis", obj)
        for mname, mfunc in _MATH.items():
            if obj is mfunc:
                return ("math", mname)
        if obj is _INLINED_FN:
            return ("inlined", None)
        if obj is compile_assert:
            return ("compile_assert", None)
        if callable(obj) and not isinstance(obj, (int, float, bool)):
            return ("pyfunc", obj)
        return ("const", obj)

    # ---------------- expressions
    def const_value(self, e):
        if e[0] == "c":
            return True, e[1]
        return False, None

    def lower_expr(self, node, env, globs, ctx):
        if isinstance(node, ast.Constant):
            return ("c", node.value)
        if isinstance(node, ast.Name):
            b = self.lookup(node.id, env, globs)
            return self.binding_expr(b, node.id)
        if isinstance(node, ast.Attribute):
            base = self.lower_obj(node.value, env, globs)
            if base[0] != "mod":
                raise SyntaxError(f"attribute access on non-module {ast.dump(node)}")
            obj = getattr(base[1], node.attr)
            b = self.classify(obj)
            return self.binding_expr(b, node.attr)
        if isinstance(node, ast.Subscript):
            b = self.lower_obj(node.value, env, globs)
            if b[0] not in ("field", "temp"):
                raise SyntaxError(f"subscript of non-field {ast.dump(node)}")
            off = self.offset_of(node.slice, env, globs, b)
            return ("f", b[1], off)
        if isinstance(node, ast.BinOp):
            a = self.lower_expr(node.left, env, globs, ctx)
            c = self.lower_expr(node.right, env, globs, ctx)
            op = _BINOPS[type(node.op)]
            ka, va = self.const_value(a)
            kc, vc = self.const_value(c)
            if ka and kc:
                return ("c", _apply_bin(op, va, vc))
            if a[0] == "axisc" and kc and op in ("+", "-"):
                return ("axisc", a[1] + vc if op == "+" else a[1] - vc)
            if c[0] == "axisc" and ka and op == "+":
                return ("axisc", c[1] + va)
            return ("bin", op, a, c)
        if isinstance(node, ast.UnaryOp):
            a = self.lower_expr(node.operand, env, globs, ctx)
            if isinstance(node.op, ast.USub):
                op = "-"
            elif isinstance(node.op, ast.UAdd):
                op = "+"
            elif isinstance(node.op, ast.Not):
                op = "not"
            else:
                raise SyntaxError(ast.dump(node))
            ka, va = self.const_value(a)
            if ka:
                return ("c", -va if op == "-" else (va if op == "+" else (not va)))
            return ("un", op, a)
        if isinstance(node, ast.Compare):
            if len(node.ops) != 1:
                raise SyntaxError("chained comparison")
            a = self.lower_expr(node.left, env, globs, ctx)
            c = self.lower_expr(node.comparators[0], env, globs, ctx)
            op = _CMPOPS[type(node.ops[0])]
            ka, va = self.const_value(a)
            kc, vc = self.const_value(c)
            if ka and kc:
                return ("c", _apply_cmp(op, va, vc))
            return ("cmp", op, a, c)
        if isinstance(node, ast.BoolOp):
            vals = [self.lower_expr(v, env, globs, ctx) for v in node.values]
            op = "and" if isinstance(node.op, ast.And) else "or"
            if all(v[0] == "c" for v in vals):
                if op == "and":
                    return ("c", all(v[1] for v in vals))
                return ("c", any(v[1] for v in vals))
            return ("bool", op, vals)
        if isinstance(node, ast.IfExp):
            cnd = self.lower_expr(node.test, env, globs, ctx)
            if cnd[0] == "c":
                branch = node.body if cnd[1] else node.orelse
                return self.lower_expr(branch, env, globs, ctx)
            a = self.lower_expr(node.body, env, globs, ctx)
            c = self.lower_expr(node.orelse, env, globs, ctx)
            return ("ifexp", cnd, a, c)
        if isinstance(node, ast.Call):
            return self.lower_call(node, env, globs, ctx)
        if isinstance(node, ast.Tuple):
            return tuple(self.lower_expr(x, env, globs, ctx) for x in node.elts)
        raise SyntaxError(f"gtscript shim: unsupported expression {ast.dump(node)}")

    def lower_obj(self, node, env, globs):
        if isinstance(node, ast.Name):
            return self.lookup(node.id, env, globs)
        if isinstance(node, ast.Attribute):
            base = self.lower_obj(node.value, env, globs)
            if base[0] != "mod":
                raise SyntaxError(ast.dump(node))
            return self.classify(getattr(base[1], node.attr))
        raise SyntaxError(ast.dump(node))

    def binding_expr(self, b, name):
        kind = b[0]
        if kind in ("field", "temp"):
            return ("f", b[1], (0, 0, 0))
        if kind == "scalar":
            return ("s", b[1])
        if kind == "const":
            return ("c", b[1])
        if kind == "axis":
            return ("axisc", b[1])
        raise SyntaxError(f"gtscript shim: {name!r} ({kind}) used as a value")

    def offset_of(self, sl, env, globs, b):
        if isinstance(sl, ast.Tuple):
            vals = []
            for n, x in enumerate(sl.elts):
                e = self.lower_expr(x, env, globs, None)
                if e[0] != "c":
                    # a vertical offset read from a field (map_single's
                    # ``q[0, 0, lev]``): a per-column gather along k
                    if n == 2 and len(sl.elts) == 3 and self.axes_of(b) == "IJK":
                        vals.append(("dyn", e))
                        continue
                    raise SyntaxError("non-constant offset")
                vals.append(int(e[1]))
        else:
            e = self.lower_expr(sl, env, globs, None)
            if e[0] != "c":
                raise SyntaxError("non-constant offset")
            vals = [int(e[1])]
        axes = self.axes_of(b)
        if axes == "IJK":
            if len(vals) == 2:
                vals = vals + [0]
            assert len(vals) == 3, vals
            return tuple(vals)
        if axes == "IJ":
            assert len(vals) in (2, 3), vals
            return (vals[0], vals[1], 0)
        if axes == "K":
            return (0, 0, vals[-1])
        if axes == "I":
            return (vals[0], 0, 0)
        if axes == "J":
            return (0, vals[0], 0)
        raise SyntaxError(f"axes {axes}")

    def axes_of(self, b):
        if b[0] == "temp":
            return "IJK"
        return self.params[b[1]][1]

    def lower_call(self, node, env, globs, ctx):
        fb = self.lower_obj(node.func, env, globs)
        kind = fb[0]
        if kind == "inlined":
            e = self.lower_expr(node.args[0], env, globs, ctx)
            if e[0] != "c":
                raise SyntaxError("__INLINED of a non-constant")
            return e
        if kind == "compile_assert":
            return ("c", True)
        if kind == "math":
            args = [self.lower_expr(a, env, globs, ctx) for a in node.args]
            if all(a[0] == "c" for a in args):
                return ("c", _apply_math(fb[1], [a[1] for a in args]))
            return ("call", fb[1], args)
        if kind == "func":
            return self.inline(fb[1], node, env, globs, ctx)
        if kind == "pyfunc" or kind == "const":
            args = [self.lower_expr(a, env, globs, ctx) for a in node.args]
            if all(a[0] == "c" for a in args):
                return ("c", fb[1](*[a[1] for a in args]))
        raise SyntaxError(f"gtscript shim: unsupported call {ast.dump(node)}")

    def inline(self, func, call, env, globs, ctx):
        fdef = _parse_function(func)
        fglobs = func.__globals__
        params = [a.arg for a in fdef.args.args]
        defaults = fdef.args.defaults
        new_env = {}
        arg_nodes = list(call.args)
        kw = {k.arg: k.value for k in call.keywords}
        for pi, pname in enumerate(params):
            if pi < len(arg_nodes):
                anode = arg_nodes[pi]
                aenv, aglobs = env, globs
            elif pname in kw:
                anode = kw[pname]
                aenv, aglobs = env, globs
            else:
                di = pi - (len(params) - len(defaults))
                anode = defaults[di]
                aenv, aglobs = {}, fglobs
            new_env[pname] = self.bind_arg(anode, aenv, aglobs, ctx)
        assigned = _assigned_names(fdef.body)
        for pname in params:
            if pname in assigned:
                src = self.binding_expr(new_env[pname], pname)
                tname = self.fresh("p")
                self.emit(tname, src, ctx)
                new_env[pname] = ("temp", tname)
        new_env["__local__"] = True
        ret = self.lower_body(fdef.body, new_env, fglobs, ctx, in_function=True)
        if ret is None:
            raise SyntaxError(f"function {func.__name__} has no return")
        return ret

    def bind_arg(self, anode, env, globs, ctx):
        if isinstance(anode, (ast.Name, ast.Attribute)):
            b = self.lower_obj(anode, env, globs)
            if b[0] in ("field", "temp", "scalar", "const", "func", "axis"):
                return b
        e = self.lower_expr(anode, env, globs, ctx)
        if e[0] == "c":
            return ("const", e[1])
        if e[0] == "s":
            return ("scalar", e[1])
        if e[0] == "f" and e[2] == (0, 0, 0):
            return ("temp", e[1]) if e[1] in self.temps else ("field", e[1])
        tname = self.fresh("a")
        self.emit(tname, e, ctx)
        return ("temp", tname)

    # ---------------- statements
    def lower_body(self, body, env, globs, ctx, in_function=False):
        ret = None
        for node in body:
            r = self.lower_stmt(node, env, globs, ctx, in_function)
            if r is not None:
                ret = r
        return ret

    def target_binding(self, name, env):
        if name in env and env[name][0] in ("field", "temp"):
            return env[name]
        if name in env and env[name][0] not in ("field", "temp"):
            # rebinding a param that held a constant/scalar
            pass
        if env.get("__local__"):
            tname = self.fresh(name)
        else:
            tname = name
            self.temps[tname] = True
        b = ("temp", tname)
        env[name] = b
        return b

    def assign(self, name, expr, env, ctx):
        if isinstance(expr, tuple) and expr and isinstance(expr[0], tuple):
            raise SyntaxError("tuple assigned to a single name")
        b = self.target_binding(name, env)
        self.emit(b[1], expr, ctx)

    def lower_stmt(self, node, env, globs, ctx, in_function):
        if isinstance(node, ast.Expr):
            if isinstance(node.value, ast.Constant):
                return None  # docstring
            if isinstance(node.value, ast.Call):
                fb = self.lower_obj(node.value.func, env, globs)
                if fb[0] == "compile_assert":
                    return None
            raise SyntaxError(f"expression statement {ast.dump(node)}")
        if isinstance(node, ast.Pass):
            return None
        if isinstance(node, ast.ImportFrom):
            if node.module == "__externals__":
                for alias in node.names:
                    val = self.externals[alias.name]
                    env[alias.asname or alias.name] = self.classify(val)
                return None
            raise SyntaxError("import inside stencil")
        if isinstance(node, ast.Return):
            val = self.lower_expr(node.value, env, globs, ctx)
            return val
        if isinstance(node, ast.Assign):
            assert len(node.targets) == 1
            tgt = node.targets[0]
            rhs = self.lower_expr(node.value, env, globs, ctx)
            if isinstance(tgt, ast.Tuple):
                names = [t.id for t in tgt.elts]
                assert isinstance(rhs, tuple) and len(rhs) == len(names)
                vals = []
                for e in rhs:
                    if e[0] == "f" and e[1] in self.temps and e[1].startswith("__"):
                        vals.append(e)
                    else:
                        tn = self.fresh("r")
                        self.emit(tn, e, ctx)
                        vals.append(("f", tn, (0, 0, 0)))
                for n, e in zip(names, vals):
                    self.assign(n, e, env, ctx)
                return None
            if isinstance(tgt, ast.Subscript):
                b = self.lower_obj(tgt.value, env, globs)
                off = self.offset_of(tgt.slice, env, globs, b)
                assert off == (0, 0, 0), "write with offset"
                self.emit(b[1], rhs, ctx)
                return None
            self.assign(tgt.id, rhs, env, ctx)
            return None
        if isinstance(node, ast.AugAssign):
            name = node.target.id
            cur = self.binding_expr(self.lookup(name, env, globs), name)
            rhs = self.lower_expr(node.value, env, globs, ctx)
            self.assign(name, ("bin", _BINOPS[type(node.op)], cur, rhs), env, ctx)
            return None
        if isinstance(node, ast.If):
            test = self.lower_expr(node.test, env, globs, ctx)
            if test[0] == "c":
                branch = node.body if test[1] else node.orelse
                return self.lower_body(branch, env, globs, ctx, in_function)
            cname = self.fresh("cond")
            self.emit(cname, test, ctx)
            cref = ("f", cname, (0, 0, 0))
            ctx_t = dict(ctx)
            ctx_t["cond"] = cref if ctx["cond"] is None else ("bool", "and", [ctx["cond"], cref])
            r1 = self.lower_body(node.body, env, globs, ctx_t, in_function)
            r2 = None
            if node.orelse:
                ncref = ("un", "not", cref)
                ctx_f = dict(ctx)
                ctx_f["cond"] = (
                    ncref if ctx["cond"] is None else ("bool", "and", [ctx["cond"], ncref])
                )
                r2 = self.lower_body(node.orelse, env, globs, ctx_f, in_function)
            if r1 is not None or r2 is not None:
                raise SyntaxError("return inside a field-dependent if")
            return None
        if isinstance(node, ast.While):
            if node.orelse:
                raise SyntaxError("while ... else")
            outer = self.cur_block
            loop = _Loop([], None, self.cur_comp, outer)
            self.cur_block = (outer[0], loop.body)
            cname = self.fresh("wcond")
            self.emit(cname, self.lower_expr(node.test, env, globs, ctx), ctx)
            cref = ("f", cname, (0, 0, 0))
            ctx_t = dict(ctx)
            ctx_t["cond"] = cref if ctx["cond"] is None else ("bool", "and", [ctx["cond"], cref])
            loop.active = ctx_t["cond"]
            r = self.lower_body(node.body, env, globs, ctx_t, in_function)
            self.cur_block = outer
            if r is not None:
                raise SyntaxError("return inside a while loop")
            outer[1].append(loop)
            return None
        if isinstance(node, ast.With):
            return self.lower_with(node, env, globs, ctx, in_function)
        raise SyntaxError(f"gtscript shim: unsupported statement {ast.dump(node)}")

    def lower_with(self, node, env, globs, ctx, in_function):
        kinds = []
        for item in node.items:
            call = item.context_expr
            assert isinstance(call, ast.Call), ast.dump(call)
            fname = call.func.id if isinstance(call.func, ast.Name) else call.func.attr
            kinds.append((fname, call))
        pushed_comp = False
        pushed_block = False
        ctx2 = dict(ctx)
        for fname, call in kinds:
            if fname == "computation":
                order_node = call.args[0]
                order = order_node.id if isinstance(order_node, ast.Name) else order_node.attr
                comp = _Comp(order)
                self.comps.append(comp)
                self.cur_comp = comp
                self.cur_block = None
                pushed_comp = True
            elif fname == "interval":
                iv = self.interval_of(call, env, globs)
                blk = (iv, [])
                self.cur_comp.blocks.append(blk)
                self.cur_block = blk
                pushed_block = True
            elif fname == "horizontal":
                regs = [self.region_of(r, env, globs) for r in call.args]
                if ctx2["regions"] is not None:
                    # nested horizontal: intersect pairwise
                    new = []
                    for a in ctx2["regions"]:
                        for b in regs:
                            new.append(_intersect_region(a, b))
                    regs = new
                ctx2["regions"] = regs
            else:
                raise SyntaxError(f"with {fname}")
        r = self.lower_body(node.body, env, globs, ctx2, in_function)
        if pushed_block:
            self.cur_block = None
        if pushed_comp:
            self.cur_comp = None
        return r

    def interval_of(self, call, env, globs):
        args = call.args
        if len(args) == 1 and isinstance(args[0], ast.Constant) and args[0].value is Ellipsis:
            return (0, None)
        vals = []
        for a in args:
            e = self.lower_expr(a, env, globs, None)
            assert e[0] == "c", ast.dump(a)
            vals.append(e[1])
        return (vals[0], vals[1])

    def region_of(self, node, env, globs):
        assert isinstance(node, ast.Subscript)
        sl = node.slice
        assert isinstance(sl, ast.Tuple) and len(sl.elts) == 2
        return tuple(self.axis_range(x, env, globs) for x in sl.elts)

    def axis_bound(self, node, env, globs):
        if node is None:
            return None
        e = self.lower_expr(node, env, globs, None)
        if e[0] == "axisc":
            return e[1]
        if e[0] == "c":
            v = int(e[1])
            return ("int", v)
        raise SyntaxError(f"region bound {ast.dump(node)}")

    def axis_range(self, node, env, globs):
        if isinstance(node, ast.Slice):
            lo = self.axis_bound(node.lower, env, globs)
            hi = self.axis_bound(node.upper, env, globs)
            return ("slice", lo, hi)
        b = self.axis_bound(node, env, globs)
        return ("index", b)


def _intersect_region(a, b):
    return ("and", a, b)


def _apply_bin(op, a, b):
    if op == "+":
        return a + b
    if op == "-":
        return a - b
    if op == "*":
        return a * b
    if op == "/":
        return a / b
    if op == "**":
        return a ** b
    if op == "%":
        return a % b
    if op == "//":
        return a // b
    raise ValueError(op)


def _apply_cmp(op, a, b):
    return {
        "<": lambda: a < b,
        "<=": lambda: a <= b,
        ">": lambda: a > b,
        ">=": lambda: a >= b,
        "==": lambda: a == b,
        "!=": lambda: a != b,
    }[op]()


def _apply_math(name, args):
    if name == "min":
        r = args[0]
        for x in args[1:]:
            r = np.minimum(r, x)
        return r
    if name == "max":
        r = args[0]
        for x in args[1:]:
            r = np.maximum(r, x)
        return r
    return _MATH[name](*args)


# ---------------------------------------------------------------- execution
_INF = 10 ** 9


def _resolve_bound(b, n, default):
    if b is None:
        return default
    if isinstance(b, AxisIndex):
        return b.resolve(n)
    assert b[0] == "int"
    v = b[1]
    return v if v >= 0 else n + v


def _range_of(r, n):
    if r[0] == "slice":
        return (_resolve_bound(r[1], n, -_INF), _resolve_bound(r[2], n, _INF))
    lo = _resolve_bound(r[1], n, None)
    return (lo, lo + 1)


def _region_boxes(region, ni, nj):
    """List of (i0, i1, j0, j1) boxes (half open) for a region spec."""
    if region[0] == "and":
        out = []
        for a in _region_boxes(region[1], ni, nj):
            for b in _region_boxes(region[2], ni, nj):
                out.append((max(a[0], b[0]), min(a[1], b[1]), max(a[2], b[2]), min(a[3], b[3])))
        return out
    ri, rj = region
    i0, i1 = _range_of(ri, ni)
    j0, j1 = _range_of(rj, nj)
    return [(i0, i1, j0, j1)]


def _box_empty(b):
    return b[0] >= b[1] or b[2] >= b[3]


def _box_intersect(a, b):
    return (max(a[0], b[0]), min(a[1], b[1]), max(a[2], b[2]), min(a[3], b[3]))


def _box_hull(a, b):
    if a is None:
        return b
    return (min(a[0], b[0]), max(a[1], b[1]), min(a[2], b[2]), max(a[3], b[3]))


def _box_contains(a, b):
    return a is not None and a[0] <= b[0] and a[1] >= b[1] and a[2] <= b[2] and a[3] >= b[3]


def _take(arr, starts, sizes):
    """arr[starts:starts+sizes] per axis, NaN where out of bounds."""
    sl = []
    ok = True
    for s, n, dim in zip(starts, sizes, arr.shape):
        if s < 0 or s + n > dim:
            ok = False
        sl.append(slice(s, s + n))
    if ok:
        return arr[tuple(sl)]
    out = np.full(sizes, np.nan)
    src, dst = [], []
    for s, n, dim in zip(starts, sizes, arr.shape):
        a0 = max(s, 0)
        a1 = min(s + n, dim)
        if a1 <= a0:
            return out
        src.append(slice(a0, a1))
        dst.append(slice(a0 - s, a1 - s))
    out[tuple(dst)] = arr[tuple(src)]
    return out


class FieldInfo:
    def __init__(self, axes, access):
        self.axes = tuple(axes)
        self.access = access


class StencilObject:
    def __init__(self, definition, externals):
        from gt4py.definitions import AccessKind

        self.definition = definition
        self.__name__ = definition.__name__
        sig = inspect.signature(definition)
        params = {}
        self.arg_names = list(sig.parameters)
        for name, p in sig.parameters.items():
            ann = p.annotation
            if isinstance(ann, FieldDescriptor):
                params[name] = ("field", ann.axes)
            else:
                params[name] = ("scalar", None)
        self.params = params
        low = _Lowering(definition, externals, params)
        fdef = _parse_function(definition)
        env = {}
        for name, (kind, _) in params.items():
            env[name] = (kind, name)
        ctx = {"cond": None, "regions": None}
        low.lower_body(fdef.body, env, definition.__globals__, ctx)
        self.comps = low.comps
        self.temps = set(low.temps)
        stmts = []

        def collect(items, ci):
            for s in items:
                if isinstance(s, _Loop):
                    s.comp = ci
                    collect(s.body, ci)
                    s.idx = s.body[0].idx
                    continue
                s.comp = ci
                s.idx = len(stmts)
                reads = []
                _expr_reads(s.expr, reads)
                if s.cond is not None:
                    _expr_reads(s.cond, reads)
                if s.cond is not None or s.regions is not None:
                    reads.append((s.target, 0, 0))
                s.reads = reads
                stmts.append(s)

        for ci, comp in enumerate(self.comps):
            for bi, (iv, blk) in enumerate(comp.blocks):
                collect(blk, ci)
        self.stmts = stmts
        written = {s.target for s in stmts}
        read = set()
        for s in stmts:
            for (n, _, _) in s.reads:
                read.add(n)
        self.field_info = {}
        for name, (kind, axes) in params.items():
            if kind != "field":
                continue
            acc = AccessKind.NONE
            if name in read:
                acc |= AccessKind.READ
            if name in written:
                acc |= AccessKind.WRITE
            self.field_info[name] = FieldInfo(axes, acc) if acc else None
        self._box_cache = {}

    # ------------------------------------------------ extent analysis
    def _boxes(self, ni, nj):
        key = (ni, nj)
        if key in self._box_cache:
            return self._box_cache[key]
        stmts = self.stmts
        boxes = [None] * len(stmts)
        writers = {}
        for s in stmts:
            writers.setdefault(s.target, []).append(s)
            if s.target not in self.temps:
                boxes[s.idx] = (0, ni, 0, nj)
        reg_cache = {}

        def regs_of(s):
            if s.regions is None:
                return None
            if s.idx not in reg_cache:
                out = []
                for r in s.regions:
                    out.extend(_region_boxes(r, ni, nj))
                reg_cache[s.idx] = out
            return reg_cache[s.idx]

        changed = True
        while changed:
            changed = False
            for t in reversed(stmts):
                bt = boxes[t.idx]
                if bt is None:
                    continue
                rl = regs_of(t)
                effs = [bt] if rl is None else [_box_intersect(bt, r) for r in rl]
                effs = [e for e in effs if not _box_empty(e)]
                if not effs:
                    continue
                seq = self.comps[t.comp].order != PARALLEL
                for (name, di, dj) in t.reads:
                    for s in writers.get(name, ()):
                        if s.idx < t.idx or (seq and s.comp == t.comp and s.idx != t.idx):
                            for e in effs:
                                need = (e[0] + di, e[1] + di, e[2] + dj, e[3] + dj)
                                if not _box_contains(boxes[s.idx], need):
                                    boxes[s.idx] = _box_hull(boxes[s.idx], need)
                                    changed = True
        self._box_cache[key] = (boxes, regs_of)
        return self._box_cache[key]

    # ------------------------------------------------ running
    def __call__(self, *args, origin=None, domain=None, validate_args=True, exec_info=None, **kwargs):
        kw = dict(zip(self.arg_names, args))
        kw.update(kwargs)
        self.run(_origin_=origin, _domain_=domain, exec_info=exec_info, **kw)

    def run(self, _origin_=None, _domain_=None, exec_info=None, **kwargs):
        ni, nj, nk = (int(x) for x in _domain_)
        origins = {}
        if isinstance(_origin_, dict):
            all_origin = _origin_.get("_all_")
        else:
            all_origin = tuple(_origin_)
            _origin_ = {}
        arrays = {}
        scalars = {}
        for name, (kind, axes) in self.params.items():
            val = kwargs[name]
            if kind == "field":
                arr = np.asarray(val)
                arrays[name] = arr
                if name in _origin_:
                    origins[name] = tuple(_origin_[name])
                else:
                    o = []
                    for ax in axes:
                        o.append(all_origin["IJK".index(ax)])
                    origins[name] = tuple(o)
            else:
                scalars[name] = val
        boxes, regs_of = self._boxes(ni, nj)
        pad = 0
        for b in boxes:
            if b is not None:
                pad = max(pad, -b[0], b[1] - ni, -b[2], b[3] - nj)
        kpad = 4
        temps = {
            t: np.full((ni + 2 * pad, nj + 2 * pad, nk + 2 * kpad), np.nan) for t in self.temps
        }
        ex = _Executor(self, arrays, origins, scalars, temps, pad, kpad, ni, nj, nk, boxes, regs_of)
        with np.errstate(all="ignore"):
            ex.execute()


class _Executor:
    def __init__(self, so, arrays, origins, scalars, temps, pad, kpad, ni, nj, nk, boxes, regs_of):
        self.so = so
        self.arrays = arrays
        self.origins = origins
        self.scalars = scalars
        self.temps = temps
        self.pad = pad
        self.kpad = kpad
        self.ni, self.nj, self.nk = ni, nj, nk
        self.boxes = boxes
        self.regs_of = regs_of

    def k_range(self, iv):
        a, b = iv
        nk = self.nk
        a = 0 if a is None else (a if a >= 0 else nk + a)
        b = nk if b is None else (b if b >= 0 else nk + b)
        return a, b

    def execute(self):
        for comp in self.so.comps:
            if comp.order == PARALLEL:
                for iv, stmts in comp.blocks:
                    k0, k1 = self.k_range(iv)
                    if k1 <= k0:
                        continue
                    for s in stmts:
                        self.exec_item(s, k0, k1)
            else:
                ranges = [(self.k_range(iv), stmts) for iv, stmts in comp.blocks]
                ks = range(self.nk) if comp.order == FORWARD else range(self.nk - 1, -1, -1)
                for k in ks:
                    for (k0, k1), stmts in ranges:
                        if k0 <= k < k1:
                            for s in stmts:
                                self.exec_item(s, k, k + 1)

    def exec_item(self, s, k0, k1):
        if not isinstance(s, _Loop):
            self.exec_stmt(s, k0, k1)
            return
        # the numpy backend's masked loop: run the body while the test holds
        # at any point of the box (bounded by the column length)
        box = self.boxes[s.body[0].idx]
        for _ in range(self.nk + 2 * self.kpad + 1):
            self.exec_stmt(s.body[0], k0, k1)
            if box is None or not np.any(_truth(self.ev(s.active, box, k0, k1))):
                return
            for b in s.body[1:]:
                self.exec_item(b, k0, k1)
        raise RuntimeError("gtscript shim: while loop did not end")

    def read(self, name, off, box, k0, k1):
        i0, i1, j0, j1 = box
        di, dj, dk = off
        if not isinstance(dk, int):
            return self.read_dyn(name, (di, dj), dk[1], box, k0, k1)
        if name in self.temps:
            p, kp = self.pad, self.kpad
            return _take(
                self.temps[name],
                (i0 + di + p, j0 + dj + p, k0 + dk + kp),
                (i1 - i0, j1 - j0, k1 - k0),
            )
        arr = self.arrays[name]
        o = self.origins[name]
        axes = self.so.params[name][1]
        if axes == "IJK":
            return _take(arr, (o[0] + i0 + di, o[1] + j0 + dj, o[2] + k0 + dk), (i1 - i0, j1 - j0, k1 - k0))
        if axes == "IJ":
            return _take(arr, (o[0] + i0 + di, o[1] + j0 + dj), (i1 - i0, j1 - j0))[:, :, None]
        if axes == "K":
            return _take(arr, (o[0] + k0 + dk,), (k1 - k0,))[None, None, :]
        if axes == "I":
            return _take(arr, (o[0] + i0 + di,), (i1 - i0,))[:, None, None]
        if axes == "J":
            return _take(arr, (o[0] + j0 + dj,), (j1 - j0,))[None, :, None]
        raise ValueError(axes)

    def read_dyn(self, name, dij, dk_expr, box, k0, k1):
        """field[i + di, j + dj, k + dk(i, j, k)] for an integer field dk."""
        i0, i1, j0, j1 = box
        di, dj = dij
        shape = (i1 - i0, j1 - j0, k1 - k0)
        dk = np.broadcast_to(np.asarray(self.ev(dk_expr, box, k0, k1)), shape).astype(np.int64)
        kk = np.arange(k0, k1)[None, None, :] + dk
        if name in self.temps:
            p, kp = self.pad, self.kpad
            arr = self.temps[name]
            plane = arr[i0 + di + p : i1 + di + p, j0 + dj + p : j1 + dj + p, :]
            kidx = kk + kp
        else:
            arr = self.arrays[name]
            o = self.origins[name]
            plane = arr[o[0] + i0 + di : o[0] + i1 + di, o[1] + j0 + dj : o[1] + j1 + dj, :]
            kidx = kk + o[2]
        ok = (kidx >= 0) & (kidx < plane.shape[2])
        out = np.take_along_axis(plane, np.clip(kidx, 0, plane.shape[2] - 1), axis=2).astype(np.float64)
        return np.where(ok, out, np.nan)

    def ev(self, e, box, k0, k1):
        tag = e[0]
        if tag == "c":
            return e[1]
        if tag == "s":
            return self.scalars[e[1]]
        if tag == "f":
            return self.read(e[1], e[2], box, k0, k1)
        if tag == "bin":
            return _apply_bin(e[1], self.ev(e[2], box, k0, k1), self.ev(e[3], box, k0, k1))
        if tag == "un":
            a = self.ev(e[2], box, k0, k1)
            if e[1] == "-":
                return -a
            if e[1] == "+":
                return a
            return np.logical_not(_truth(a))
        if tag == "cmp":
            return _apply_cmp(e[1], self.ev(e[2], box, k0, k1), self.ev(e[3], box, k0, k1))
        if tag == "bool":
            vals = [_truth(self.ev(x, box, k0, k1)) for x in e[2]]
            r = vals[0]
            for v in vals[1:]:
                r = np.logical_and(r, v) if e[1] == "and" else np.logical_or(r, v)
            return r
        if tag == "ifexp":
            c = _truth(self.ev(e[1], box, k0, k1))
            return np.where(c, self.ev(e[2], box, k0, k1), self.ev(e[3], box, k0, k1))
        if tag == "call":
            return _apply_math(e[1], [self.ev(a, box, k0, k1) for a in e[2]])
        raise ValueError(tag)

    def exec_stmt(self, s, k0, k1):
        box = self.boxes[s.idx]
        if box is None:
            return
        shape = (box[1] - box[0], box[3] - box[2], k1 - k0)
        mask = None
        rl = self.regs_of(s)
        if rl is not None:
            m2 = np.zeros(shape[:2], dtype=bool)
            any_in = False
            for r in rl:
                rb = _box_intersect(box, r)
                if _box_empty(rb):
                    continue
                any_in = True
                m2[rb[0] - box[0] : rb[1] - box[0], rb[2] - box[2] : rb[3] - box[2]] = True
            if not any_in:
                return
            mask = np.broadcast_to(m2[:, :, None], shape)
        if s.cond is not None:
            c = np.broadcast_to(_truth(self.ev(s.cond, box, k0, k1)), shape)
            mask = c if mask is None else np.logical_and(mask, c)
        val = self.ev(s.expr, box, k0, k1)
        if isinstance(val, (bool, np.bool_)) or (isinstance(val, np.ndarray) and val.dtype == bool):
            val = np.asarray(val, dtype=np.float64)
        val = np.broadcast_to(np.asarray(val, dtype=np.float64), shape)
        self.write(s.target, box, k0, k1, val, mask)

    def write(self, name, box, k0, k1, val, mask):
        i0, i1, j0, j1 = box
        if name in self.temps:
            p, kp = self.pad, self.kpad
            view = self.temps[name][i0 + p : i1 + p, j0 + p : j1 + p, k0 + kp : k1 + kp]
        else:
            arr = self.arrays[name]
            o = self.origins[name]
            axes = self.so.params[name][1]
            if axes == "IJK":
                a0, a1 = o[0] + i0, o[0] + i1
                b0, b1 = o[1] + j0, o[1] + j1
                c0, c1 = o[2] + k0, o[2] + k1
                # clip to the storage (writes outside the allocation are dropped)
                ci0, ci1 = max(a0, 0), min(a1, arr.shape[0])
                cj0, cj1 = max(b0, 0), min(b1, arr.shape[1])
                ck0, ck1 = max(c0, 0), min(c1, arr.shape[2])
                if ci1 <= ci0 or cj1 <= cj0 or ck1 <= ck0:
                    return
                view = arr[ci0:ci1, cj0:cj1, ck0:ck1]
                sl = (slice(ci0 - a0, ci1 - a0), slice(cj0 - b0, cj1 - b0), slice(ck0 - c0, ck1 - c0))
                val = val[sl]
                if mask is not None:
                    mask = mask[sl]
            elif axes == "IJ":
                a0, a1 = o[0] + i0, o[0] + i1
                b0, b1 = o[1] + j0, o[1] + j1
                ci0, ci1 = max(a0, 0), min(a1, arr.shape[0])
                cj0, cj1 = max(b0, 0), min(b1, arr.shape[1])
                view = arr[ci0:ci1, cj0:cj1]
                sl = (slice(ci0 - a0, ci1 - a0), slice(cj0 - b0, cj1 - b0))
                val = val[sl][:, :, -1]
                if mask is not None:
                    mask = mask[sl][:, :, -1]
            elif axes == "K":
                view = arr[o[0] + k0 : o[0] + k1]
                val = val[0, 0, :]
                if mask is not None:
                    mask = mask[0, 0, :]
            else:
                raise ValueError(axes)
        if mask is None:
            view[...] = val
        else:
            view[...] = np.where(mask, val, view)


def _truth(a):
    if isinstance(a, np.ndarray):
        if a.dtype == bool:
            return a
        return a != 0
    return bool(a)


def stencil(definition=None, *, backend=None, externals=None, rebuild=False, **kwargs):
    def build(defn):
        return StencilObject(defn, externals or {})

    if definition is None:
        return build
    return build(definition)
