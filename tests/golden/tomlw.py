"""A minimal TOML writer for Yuzen case files (tables of scalars, strings and
flat arrays), used to write variants of the reference's cases."""
from __future__ import annotations


def _val(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        return repr(v)
    if isinstance(v, str):
        return '"' + v.replace("\\", "\\\\").replace('"', '\\"') + '"'
    if isinstance(v, (list, tuple)):
        return "[" + ", ".join(_val(x) for x in v) + "]"
    raise TypeError(f"cannot write {type(v)}")


def dumps(doc: dict) -> str:
    lines: list[str] = []

    def emit(table: dict, prefix: str) -> None:
        scalars = [(k, v) for k, v in table.items() if not isinstance(v, dict)]
        subs = [(k, v) for k, v in table.items() if isinstance(v, dict)]
        if prefix:
            lines.append(f"[{prefix}]")
        for k, v in scalars:
            lines.append(f"{k} = {_val(v)}")
        if prefix or scalars:
            lines.append("")
        for k, v in subs:
            emit(v, f"{prefix}.{k}" if prefix else k)

    emit(doc, "")
    return "\n".join(lines) + "\n"


def setpath(doc: dict, path: str, value) -> None:
    keys = path.split(".")
    cur = doc
    for k in keys[:-1]:
        cur = cur.setdefault(k, {})
    cur[keys[-1]] = value
