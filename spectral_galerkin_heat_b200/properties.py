"""Temperature-dependent material properties and their device bytecode.

Mirrors the reference's property model: the whitelisted expression grammar of
``core/property_expr.py`` (:53-157, names ``T``, ``pi``, ``e``; ``+ - * / **``;
unary ``+``/``-``; the function list of ``_NUMPY_FUNC_NAME`` :68-76),
``liquid_fraction`` / ``TempProperty`` / ``MaterialModel`` of
``core/properties.py`` (:61-150, :242-479).

The reference turns each expression into generated CUDA-C compiled at run
time. Here every expression is compiled once, on the host, into a short
postfix program (``SGH_OP_*`` opcodes of ``include/sgh_b200.h``) that the
kernels interpret per cell. All threads of a launch run the same program, so
the interpreter loop is warp-uniform; operations are applied in the same order
as the Python evaluation of the tree, which keeps FP64 results equal to the
host evaluation up to the last-ulp differences of the transcendental functions.
"""
from __future__ import annotations

import ast
import math
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np

__all__ = ["PropertyExpr", "TempProperty", "MaterialModel", "liquid_fraction",
           "OPCODES", "MAX_PROGRAM", "MAX_STACK"]

# Opcode numbers; must match the SGH_OP_* enum in include/sgh_b200.h.
OPCODES = {
    "const": 1, "T": 2, "add": 3, "sub": 4, "mul": 5, "div": 6, "pow": 7, "neg": 8,
    "sqrt": 16, "exp": 17, "log": 18, "log2": 19, "log10": 20, "sin": 21, "cos": 22,
    "tan": 23, "asin": 24, "acos": 25, "atan": 26, "sinh": 27, "cosh": 28, "tanh": 29,
    "asinh": 30, "acosh": 31, "atanh": 32, "fabs": 33, "ceil": 34, "floor": 35,
    "trunc": 36, "log1p": 37, "expm1": 38, "atan2": 48,
}
MAX_PROGRAM = 64   # instructions per expression (SGH_MAX_PROGRAM)
MAX_STACK = 16     # evaluation stack depth (SGH_MAX_STACK)

_NUMPY_NAME = {
    "sqrt": "sqrt", "exp": "exp", "log": "log", "log2": "log2", "log10": "log10",
    "sin": "sin", "cos": "cos", "tan": "tan", "asin": "arcsin", "acos": "arccos",
    "atan": "arctan", "atan2": "arctan2", "sinh": "sinh", "cosh": "cosh", "tanh": "tanh",
    "asinh": "arcsinh", "acosh": "arccosh", "atanh": "arctanh", "fabs": "abs",
    "ceil": "ceil", "floor": "floor", "trunc": "trunc", "log1p": "log1p", "expm1": "expm1",
}
_CONSTANTS = {"pi": math.pi, "e": math.e}


def _check(node) -> None:
    if isinstance(node, ast.Constant):
        if isinstance(node.value, bool) or not isinstance(node.value, (int, float)):
            raise ValueError(f"Only numeric literals are allowed, got {node.value!r}.")
    elif isinstance(node, ast.Name):
        if node.id != "T" and node.id not in _CONSTANTS:
            raise ValueError(f"Unknown name {node.id!r} in property expression "
                             f"(only 'T' and {sorted(_CONSTANTS)} are allowed).")
    elif isinstance(node, ast.BinOp):
        if not isinstance(node.op, (ast.Add, ast.Sub, ast.Mult, ast.Div, ast.Pow)):
            raise ValueError(f"Operator {type(node.op).__name__} is not allowed.")
        _check(node.left)
        _check(node.right)
    elif isinstance(node, ast.UnaryOp):
        if not isinstance(node.op, (ast.UAdd, ast.USub)):
            raise ValueError(f"Unary operator {type(node.op).__name__} is not allowed.")
        _check(node.operand)
    elif isinstance(node, ast.Call):
        if (not isinstance(node.func, ast.Name) or node.func.id not in _NUMPY_NAME
                or node.keywords or not node.args):
            raise ValueError(f"Function {getattr(node.func, 'id', '<expr>')!r} is not "
                             "allowed in a property expression.")
        want = 2 if node.func.id == "atan2" else 1
        if len(node.args) != want:
            raise ValueError(f"{node.func.id} takes {want} argument(s).")
        for a in node.args:
            _check(a)
    else:
        raise ValueError(f"{type(node).__name__} is not allowed in a property expression.")


class PropertyExpr:
    """A validated expression of ``T`` (or a bare constant)."""

    __slots__ = ("source", "_const", "_tree")

    def __init__(self, expr):
        self.source = str(expr).strip()
        try:
            self._const = float(self.source)
            self._tree = None
            return
        except ValueError:
            pass
        try:
            tree = ast.parse(self.source, mode="eval").body
        except SyntaxError as exc:
            raise ValueError(f"Invalid property expression {self.source!r}: {exc}") from None
        _check(tree)
        self._const, self._tree = None, tree

    @property
    def is_constant(self) -> bool:
        return self._const is not None

    @property
    def constant_value(self) -> float:
        if self._const is None:
            raise ValueError(f"{self.source!r} is not a constant expression.")
        return self._const

    def __call__(self, T):
        if self._const is not None:
            return T * 0.0 + self._const
        return _evaluate(self._tree, T)

    def program(self) -> tuple[list[int], list[float]]:
        """Postfix program ``(ops, consts)``: ``ops`` holds opcode numbers, and
        each ``const`` opcode is followed by the index of its value in ``consts``."""
        ops: list[int] = []
        consts: list[float] = []
        if self._const is not None:
            ops += [OPCODES["const"], 0]
            consts.append(self._const)
        else:
            _emit(self._tree, ops, consts)
        if len(ops) > MAX_PROGRAM:
            raise ValueError(f"Property expression {self.source!r} is too long for the "
                             f"device interpreter ({len(ops)} > {MAX_PROGRAM} slots).")
        if _stack_depth(ops) > MAX_STACK:
            raise ValueError(f"Property expression {self.source!r} nests too deeply.")
        return ops, consts

    def __repr__(self):
        return f"PropertyExpr({self.source!r})"


def _evaluate(node, T):
    if isinstance(node, ast.Constant):
        return node.value
    if isinstance(node, ast.Name):
        return T if node.id == "T" else _CONSTANTS[node.id]
    if isinstance(node, ast.BinOp):
        a, b = _evaluate(node.left, T), _evaluate(node.right, T)
        op = type(node.op)
        if op is ast.Add:
            return a + b
        if op is ast.Sub:
            return a - b
        if op is ast.Mult:
            return a * b
        if op is ast.Div:
            return a / b
        return a ** b
    if isinstance(node, ast.UnaryOp):
        v = _evaluate(node.operand, T)
        return -v if isinstance(node.op, ast.USub) else v
    fn = getattr(np, _NUMPY_NAME[node.func.id])
    return fn(*(_evaluate(a, T) for a in node.args))


def _emit(node, ops, consts) -> None:
    if isinstance(node, ast.Constant):
        ops += [OPCODES["const"], len(consts)]
        consts.append(float(node.value))
    elif isinstance(node, ast.Name):
        if node.id == "T":
            ops.append(OPCODES["T"])
        else:
            ops += [OPCODES["const"], len(consts)]
            consts.append(_CONSTANTS[node.id])
    elif isinstance(node, ast.BinOp):
        _emit(node.left, ops, consts)
        _emit(node.right, ops, consts)
        ops.append(OPCODES[{ast.Add: "add", ast.Sub: "sub", ast.Mult: "mul",
                            ast.Div: "div", ast.Pow: "pow"}[type(node.op)]])
    elif isinstance(node, ast.UnaryOp):
        _emit(node.operand, ops, consts)
        if isinstance(node.op, ast.USub):
            ops.append(OPCODES["neg"])
    else:
        for a in node.args:
            _emit(a, ops, consts)
        ops.append(OPCODES[node.func.id])


def _stack_depth(ops) -> int:
    depth = peak = 0
    i = 0
    while i < len(ops):
        op = ops[i]
        if op == OPCODES["const"]:
            depth += 1
            i += 2
            peak = max(peak, depth)
            continue
        if op == OPCODES["T"]:
            depth += 1
        elif op in (3, 4, 5, 6, 7, OPCODES["atan2"]):
            depth -= 1
        peak = max(peak, depth)
        i += 1
    return peak


def liquid_fraction(T, T_solidus, T_liquidus):
    """``clip((T - T_s)/(T_l - T_s), 0, 1)``; a step at ``T_s`` when ``T_l <= T_s``."""
    if T_liquidus <= T_solidus:
        if hasattr(T, "shape"):
            return np.where(np.asarray(T) >= T_solidus, 1.0, 0.0).astype(T.dtype)
        return 1.0 if T >= T_solidus else 0.0
    f = (T - T_solidus) / (T_liquidus - T_solidus)
    if hasattr(f, "clip"):
        return f.clip(0.0, 1.0)
    return min(max(f, 0.0), 1.0)


@dataclass
class TempProperty:
    """One property with solid and liquid branches blended by the liquid fraction."""

    solid: PropertyExpr
    liquid: PropertyExpr
    T_solidus: float
    T_liquidus: float
    is_constant: bool = False

    def __call__(self, T):
        if self.is_constant:
            return self.solid(T)
        fl = liquid_fraction(T, self.T_solidus, self.T_liquidus)
        return (1.0 - fl) * self.solid(T) + fl * self.liquid(T)

    @classmethod
    def from_config(cls, spec: Any, T_solidus: float, T_liquidus: float) -> "TempProperty":
        if isinstance(spec, dict) and ("solid" in spec or "liquid" in spec):
            solid = PropertyExpr(spec.get("solid", spec.get("liquid")))
            liquid = PropertyExpr(spec.get("liquid", spec.get("solid")))
            const = (solid.is_constant and liquid.is_constant
                     and solid.constant_value == liquid.constant_value)
            return cls(solid, liquid, float(T_solidus), float(T_liquidus), const)
        value = spec["value"] if isinstance(spec, dict) else spec
        c = PropertyExpr(value)
        return cls(c, c, float(T_solidus), float(T_liquidus), True)


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
        return self.k.is_constant and self.rho.is_constant and self.c.is_constant

    def recommended_references(self, T_lo: float, T_hi: float, n_samples: int = 512):
        """Midpoint of each property's extrema over ``[T_lo, T_hi]`` -> ``(k, rho, Cp)``."""
        T = np.linspace(float(T_lo), float(T_hi), int(n_samples))

        def mid(p):
            v = np.asarray(p(T), dtype=np.float64)
            return 0.5 * (float(v.min()) + float(v.max()))

        return mid(self.k), mid(self.rho), mid(self.c)

    @classmethod
    def from_config(cls, mat_cfg: dict, T_solidus: float, T_liquidus: float
                    ) -> Optional["MaterialModel"]:
        def branched(s):
            return isinstance(s, dict) and ("solid" in s or "liquid" in s)

        specs = {"k": mat_cfg.get("k"), "rho": mat_cfg.get("rho"), "c": mat_cfg.get("Cp")}
        if not any(branched(s) for s in specs.values()):
            return None
        return cls(k=TempProperty.from_config(specs["k"], T_solidus, T_liquidus),
                   rho=TempProperty.from_config(specs["rho"], T_solidus, T_liquidus),
                   c=TempProperty.from_config(specs["c"], T_solidus, T_liquidus))
