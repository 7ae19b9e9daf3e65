"""Write a problem, given as nested Python dicts, in the libconfig text format
of the reference's ``inputParam.cfg`` (src/GeneralModel/inputParam.cfg).

Type mapping follows libconfig: Python ``float`` -> float literal (always with
a '.' or an exponent, because the reference reads real-valued settings with
strict typing, e.g. ``ncycles = 8.``), ``int`` -> integer, ``bool`` ->
true/false, ``str`` -> quoted string, a list of scalars -> array ``[...]``, a
list of dicts -> list ``( {...}, ... )``, a dict -> group ``{...}``.
"""
from __future__ import annotations


def _scalar(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        r = repr(v)
        if r in ("inf", "-inf", "nan"):
            raise ValueError("libconfig has no literal for " + r)
        if "." not in r and "e" not in r and "E" not in r:
            r += ".0"
        return r
    if isinstance(v, str):
        return '"' + v.replace("\\", "\\\\").replace('"', '\\"') + '"'
    raise TypeError(f"cannot write {type(v).__name__} as a libconfig scalar")


def _value(v, indent: str) -> str:
    if isinstance(v, dict):
        inner = indent + "    "
        body = "".join(f"{inner}{k} = {_value(x, inner)};\n" for k, x in v.items())
        return "{\n" + body + indent + "}"
    if isinstance(v, (list, tuple)):
        if v and all(isinstance(x, dict) for x in v):
            inner = indent + "    "
            return "(\n" + ",\n".join(inner + _value(x, inner) for x in v) + "\n" + indent + ")"
        return "[" + ", ".join(_scalar(x) for x in v) + "]"
    return _scalar(v)


def dumps(case: dict) -> str:
    """Return the libconfig text of ``case`` (top-level settings in order)."""
    return "".join(f"{k} = {_value(v, '')};\n" for k, v in case.items())
