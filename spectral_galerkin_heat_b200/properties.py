"""Temperature-dependent material properties, compiled to device bytecode.

The configuration language is the reference's (``core/property_expr.py:53-157``
defines the grammar; ``core/properties.py:61-150, 242-479`` the solid/liquid
model): a property branch is a number or an expression of ``T`` built from
numeric literals, the names ``T``, ``pi`` and ``e``, the operators
``+ - * / **``, unary ``+``/``-`` and calls of a fixed list of one-argument
math functions (two for ``atan2``). Config files written for the reference
therefore parse to the same properties here.

The implementation is this library's own. An expression is lowered in one
pass, straight from Python's syntax tree, into the postfix program that the
CUDA kernels interpret per cell (``SGH_OP_*`` opcodes of
``include/sgh_b200.h``, ``eval_program`` in ``csrc/sgh_device.cuh``). Every
node kind has one lowering rule in a dispatch table; a node kind with no rule,
or a rule that refuses its node, is a ``ValueError`` raised while lowering, so
validation and compilation are the same walk. Host-side values
(``PropertyExpr.__call__``, the reference constants, the recommended
references) come from :class:`Program.run`, a NumPy stack machine that executes
the very program the device runs, in the same operation order.
"""
from __future__ import annotations

import ast
import math
from dataclasses import dataclass
from typing import Any, Callable, Optional

import numpy as np

__all__ = ["PropertyExpr", "TempProperty", "MaterialModel", "Program", "liquid_fraction",
           "compile_expression", "OPCODES", "MAX_PROGRAM", "MAX_STACK"]

# Opcode numbers; must match the SGH_OP_* enum in include/sgh_b200.h.
OPCODES = {
    "const": 1, "T": 2, "add": 3, "sub": 4, "mul": 5, "div": 6, "pow": 7, "neg": 8,
    "sqrt": 16, "exp": 17, "log": 18, "log2": 19, "log10": 20, "sin": 21, "cos": 22,
    "tan": 23, "asin": 24, "acos": 25, "atan": 26, "sinh": 27, "cosh": 28, "tanh": 29,
    "asinh": 30, "acosh": 31, "atanh": 32, "fabs": 33, "ceil": 34, "floor": 35,
    "trunc": 36, "log1p": 37, "expm1": 38, "atan2": 48,
}
MAX_PROGRAM = 64   # instruction slots per expression (SGH_MAX_PROGRAM)
MAX_STACK = 16     # evaluation stack depth (SGH_MAX_STACK)

# Host semantics of every opcode: (arity, numpy implementation).
_HOST_OP: dict[int, tuple[int, Callable]] = {
    OPCODES["add"]: (2, np.add), OPCODES["sub"]: (2, np.subtract),
    OPCODES["mul"]: (2, np.multiply), OPCODES["div"]: (2, np.true_divide),
    OPCODES["pow"]: (2, np.power), OPCODES["atan2"]: (2, np.arctan2),
    OPCODES["neg"]: (1, np.negative),
    OPCODES["sqrt"]: (1, np.sqrt), OPCODES["exp"]: (1, np.exp), OPCODES["log"]: (1, np.log),
    OPCODES["log2"]: (1, np.log2), OPCODES["log10"]: (1, np.log10),
    OPCODES["sin"]: (1, np.sin), OPCODES["cos"]: (1, np.cos), OPCODES["tan"]: (1, np.tan),
    OPCODES["asin"]: (1, np.arcsin), OPCODES["acos"]: (1, np.arccos),
    OPCODES["atan"]: (1, np.arctan), OPCODES["sinh"]: (1, np.sinh),
    OPCODES["cosh"]: (1, np.cosh), OPCODES["tanh"]: (1, np.tanh),
    OPCODES["asinh"]: (1, np.arcsinh), OPCODES["acosh"]: (1, np.arccosh),
    OPCODES["atanh"]: (1, np.arctanh), OPCODES["fabs"]: (1, np.abs),
    OPCODES["ceil"]: (1, np.ceil), OPCODES["floor"]: (1, np.floor),
    OPCODES["trunc"]: (1, np.trunc), OPCODES["log1p"]: (1, np.log1p),
    OPCODES["expm1"]: (1, np.expm1),
}
# Callable names of the grammar -> opcode; the operand count is in _HOST_OP.
_CALLS = {name: OPCODES[name] for name in (
    "sqrt", "exp", "log", "log2", "log10", "sin", "cos", "tan", "asin", "acos", "atan",
    "atan2", "sinh", "cosh", "tanh", "asinh", "acosh", "atanh", "fabs", "ceil", "floor",
    "trunc", "log1p", "expm1")}
_NAMED_CONSTANTS = {"pi": math.pi, "e": math.e}
_BINARY = {ast.Add: "add", ast.Sub: "sub", ast.Mult: "mul", ast.Div: "div", ast.Pow: "pow"}


@dataclass(frozen=True)
class Program:
    """A postfix program: ``ops`` holds opcode numbers, and every ``const``
    opcode is followed by the index of its value in ``consts``."""

    ops: tuple
    consts: tuple

    @property
    def max_depth(self) -> int:
        """Deepest evaluation stack the program needs."""
        depth = peak = 0
        for op, _ in self._decode():
            if op in (OPCODES["const"], OPCODES["T"]):
                depth += 1
            else:
                depth -= _HOST_OP[op][0] - 1
            peak = max(peak, depth)
        return peak

    def _decode(self):
        i = 0
        while i < len(self.ops):
            op = self.ops[i]
            if op == OPCODES["const"]:
                yield op, self.consts[self.ops[i + 1]]
                i += 2
            else:
                yield op, None
                i += 1

    def run(self, T):
        """Execute on a scalar or an array of temperatures (float64)."""
        T = np.asarray(T, dtype=np.float64) if not np.isscalar(T) else float(T)
        stack: list = []
        for op, value in self._decode():
            if op == OPCODES["const"]:
                stack.append(value)
            elif op == OPCODES["T"]:
                stack.append(T)
            else:
                arity, fn = _HOST_OP[op]
                args = stack[-arity:]
                del stack[-arity:]
                stack.append(fn(*args))
        (out,) = stack
        # a program without T still yields one value per temperature
        return out + np.zeros_like(T) if np.ndim(T) else out


class _Lowering:
    """One expression's lowering into a :class:`Program` (single use)."""

    def __init__(self, source: str):
        self.source = source
        self.ops: list[int] = []
        self.consts: list[float] = []

    def fail(self, what: str):
        raise ValueError(f"property expression {self.source!r}: {what}")

    def emit_const(self, value: float):
        self.ops += [OPCODES["const"], len(self.consts)]
        self.consts.append(float(value))

    def lower(self, node):
        rule = self.RULES.get(type(node))
        if rule is None:
            self.fail(f"{type(node).__name__} nodes are outside the property grammar")
        rule(self, node)

    def _constant(self, node):
        v = node.value
        if isinstance(v, bool) or not isinstance(v, (int, float)):
            self.fail(f"literal {v!r} is not a real number")
        self.emit_const(v)

    def _name(self, node):
        if node.id == "T":
            self.ops.append(OPCODES["T"])
        elif node.id in _NAMED_CONSTANTS:
            self.emit_const(_NAMED_CONSTANTS[node.id])
        else:
            self.fail(f"name {node.id!r} is undefined; the variable is 'T' and the "
                      f"constants are {sorted(_NAMED_CONSTANTS)}")

    def _binary(self, node):
        op = _BINARY.get(type(node.op))
        if op is None:
            self.fail(f"operator {type(node.op).__name__} is outside the property grammar")
        self.lower(node.left)
        self.lower(node.right)
        self.ops.append(OPCODES[op])

    def _unary(self, node):
        if isinstance(node.op, ast.UAdd):
            self.lower(node.operand)
        elif isinstance(node.op, ast.USub):
            self.lower(node.operand)
            self.ops.append(OPCODES["neg"])
        else:
            self.fail(f"unary operator {type(node.op).__name__} is outside the property grammar")

    def _call(self, node):
        name = node.func.id if isinstance(node.func, ast.Name) else None
        if name not in _CALLS:
            self.fail(f"call of {ast.unparse(node.func)!r} is outside the property grammar")
        if node.keywords:
            self.fail(f"{name}() takes positional arguments only")
        arity = _HOST_OP[_CALLS[name]][0]
        if len(node.args) != arity:
            self.fail(f"{name}() takes {arity} argument(s), got {len(node.args)}")
        for arg in node.args:
            self.lower(arg)
        self.ops.append(_CALLS[name])

    RULES = {ast.Constant: _constant, ast.Name: _name, ast.BinOp: _binary,
             ast.UnaryOp: _unary, ast.Call: _call}


def compile_expression(source) -> Program:
    """Lower a property expression (or a bare number) to a device :class:`Program`."""
    text = str(source).strip()
    low = _Lowering(text)
    try:
        low.emit_const(float(text))
    except ValueError:
        try:
            tree = ast.parse(text, mode="eval")
        except SyntaxError as exc:
            raise ValueError(f"property expression {text!r} does not parse: {exc.msg}") from None
        low.lower(tree.body)
    prog = Program(tuple(low.ops), tuple(low.consts))
    if len(prog.ops) > MAX_PROGRAM:
        raise ValueError(f"property expression {text!r} needs {len(prog.ops)} program slots; "
                         f"the device interpreter holds {MAX_PROGRAM}")
    if prog.max_depth > MAX_STACK:
        raise ValueError(f"property expression {text!r} nests deeper than the device "
                         f"stack ({MAX_STACK})")
    return prog


class PropertyExpr:
    """A property branch: a number or an expression of ``T``, held as its program."""

    __slots__ = ("source", "_prog", "_number")

    def __init__(self, expr):
        self.source = str(expr).strip()
        self._prog = compile_expression(self.source)
        try:
            self._number = float(self.source)
        except ValueError:
            self._number = None

    @property
    def is_constant(self) -> bool:
        """True for a bare number (an expression without ``T`` still counts as
        an expression, as in the reference)."""
        return self._number is not None

    @property
    def constant_value(self) -> float:
        if self._number is None:
            raise ValueError(f"{self.source!r} is an expression, not a number")
        return self._number

    def __call__(self, T):
        return self._prog.run(T)

    def program(self) -> tuple[list[int], list[float]]:
        """``(ops, consts)`` of the device program."""
        return list(self._prog.ops), list(self._prog.consts)

    def __repr__(self):
        return f"PropertyExpr({self.source!r})"


def liquid_fraction(T, T_solidus, T_liquidus):
    """Liquid fraction: a linear ramp from 0 at the solidus to 1 at the liquidus,
    or a step at the solidus when the band is empty (``T_liquidus <= T_solidus``).
    Arrays keep their dtype; scalars give a float."""
    Ts, Tl = float(T_solidus), float(T_liquidus)
    arr = np.asarray(T)
    if Tl > Ts:
        f = np.clip((arr - Ts) / (Tl - Ts), 0.0, 1.0)
    else:
        f = (arr >= Ts).astype(arr.dtype if arr.dtype.kind == "f" else np.float64)
    return f if np.ndim(T) else float(f)


@dataclass
class TempProperty:
    """One property: solid and liquid branches blended by the liquid fraction,
    ``p(T) = (1 - f_l) p_solid(T) + f_l p_liquid(T)``. ``is_constant`` marks a
    property whose branches are the same number (the constant-coefficient path)."""

    solid: PropertyExpr
    liquid: PropertyExpr
    T_solidus: float
    T_liquidus: float
    is_constant: bool = False

    def __call__(self, T):
        if self.is_constant:
            return self.solid(T)
        f = liquid_fraction(T, self.T_solidus, self.T_liquidus)
        return (1.0 - f) * self.solid(T) + f * self.liquid(T)

    @staticmethod
    def _branches(spec) -> Optional[tuple]:
        """``(solid, liquid)`` sources of a branch mapping (one missing branch
        takes the other), or None for a scalar spec."""
        if not isinstance(spec, dict):
            return None
        present = [spec[k] for k in ("solid", "liquid") if k in spec]
        if not present:
            return None
        return spec.get("solid", present[0]), spec.get("liquid", present[0])

    @classmethod
    def from_config(cls, spec: Any, T_solidus: float, T_liquidus: float) -> "TempProperty":
        """From a number, a ``{value, unit}`` mapping or a ``{solid, liquid}``
        mapping (whose ``reference``/``unit`` keys the config parser reads)."""
        band = (float(T_solidus), float(T_liquidus))
        branches = cls._branches(spec)
        if branches is None:
            c = PropertyExpr(spec["value"] if isinstance(spec, dict) else spec)
            return cls(c, c, *band, is_constant=True)
        s, l = PropertyExpr(branches[0]), PropertyExpr(branches[1])
        same = s.is_constant and l.is_constant and s.constant_value == l.constant_value
        return cls(s, l, *band, is_constant=same)


# config key -> MaterialModel field
_MODEL_FIELDS = (("k", "k"), ("rho", "rho"), ("Cp", "c"))


@dataclass
class MaterialModel:
    """``k(T)``, ``rho(T)``, ``c(T)``; ``a(T) = rho(T) c(T)``."""

    k: TempProperty
    rho: TempProperty
    c: TempProperty

    def a(self, T):
        return self.rho(T) * self.c(T)

    @property
    def is_constant(self) -> bool:
        return all(getattr(self, f).is_constant for _, f in _MODEL_FIELDS)

    def by_config_key(self, key: str) -> TempProperty:
        """The property of config key ``k`` / ``rho`` / ``Cp``."""
        return getattr(self, dict(_MODEL_FIELDS)[key])

    def recommended_references(self, T_lo: float, T_hi: float, n_samples: int = 512):
        """``(k, rho, Cp)`` reference constants: for each property the midpoint of
        its smallest and largest value on ``n_samples`` points of ``[T_lo, T_hi]``."""
        T = np.linspace(float(T_lo), float(T_hi), int(n_samples))
        out = []
        for _, f in _MODEL_FIELDS:
            v = np.asarray(getattr(self, f)(T), dtype=np.float64)
            out.append(0.5 * (float(v.min()) + float(v.max())))
        return tuple(out)

    @classmethod
    def from_config(cls, mat_cfg: dict, T_solidus: float, T_liquidus: float
                    ) -> Optional["MaterialModel"]:
        """The model of a material section, or None when no property has branches."""
        specs = {key: mat_cfg.get(key) for key, _ in _MODEL_FIELDS}
        if all(TempProperty._branches(s) is None for s in specs.values()):
            return None
        return cls(**{f: TempProperty.from_config(specs[key], T_solidus, T_liquidus)
                      for key, f in _MODEL_FIELDS})
