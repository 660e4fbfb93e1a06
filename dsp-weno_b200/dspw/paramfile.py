"""Writer and reader for the reference's ``param.in`` surface.

The grammar is the one read by ``Parameter::read`` in the reference
(enflo/src/parameter.cc:16-29 for systems, enflo_scalar/src_scalar/parameter.cc for
scalar laws): sections ``grid``, ``numeric``, ``material``, ``constants``,
``initial_condition``, ``exact_soln``, ``boundary_condition`` and ``output``,
entries separated by whitespace, ``#``/``%``/``//`` line comments and ``/* */``
block comments (enflo/src/reader.h:49-88).

``write_param`` produces a file from a plain dict so tests, the benchmark and
users can generate cases without hand-editing text.  ``read_param`` is a small
tokenizer used by the Python side to inspect a file; the C++ host driver has
its own reader.
"""
from __future__ import annotations

import re

_BC_NAMES = ("xleft", "xright", "yleft", "yright", "zleft", "zright")


def _levels(v):
    if isinstance(v, (list, tuple)):
        return "{ " + ",".join(str(int(x)) for x in v) + " }"
    return "{ %d }" % int(v)


def write_param(cfg: dict) -> str:
    """Return param.in text for ``cfg``.

    Keys (defaults in brackets): ``model`` (linadv | burgers | euler | ns_es |
    ns_kep), ``x``/``y``/``z`` = (min, max) as numbers or expressions,
    ``Nx``/``Ny``/``Nz`` (int or list for OOC levels), ``cfl``, ``final_time``,
    ``max_iter`` [50000], ``reconstruct`` [sp_weno], ``net_file`` [none],
    ``flux``, ``vel`` (linadv, 3 numbers), ``gamma`` [1.4], ``gas_const`` [1],
    ``mu_ref`` [0], ``prandtl`` [1], ``EC1_fix`` [no], ``constants`` (dict),
    ``ic`` (scalar: str; systems: dict density/xvelocity/yvelocity/zvelocity/
    pressure), ``exact`` (same shape or None), ``bc`` (6 names or one name),
    ``ooc`` [no], ``dim`` [1], ``time_stamps`` [1], ``output_path`` [.].
    """
    model = cfg["model"]
    scalar = model in ("linadv", "burgers")
    x0, x1 = cfg.get("x", (0, 1))
    y0, y1 = cfg.get("y", (0, 1))
    z0, z1 = cfg.get("z", (0, 1))
    out = []
    out.append("grid\n{")
    out.append(f"   x_min   {x0}\n   x_max   {x1}\n   Nx_cell {_levels(cfg['Nx'])}")
    out.append(f"   y_min   {y0}\n   y_max   {y1}\n   Ny_cell {_levels(cfg.get('Ny', 2))}")
    out.append(f"   z_min   {z0}\n   z_max   {z1}\n   Nz_cell {_levels(cfg.get('Nz', 2))}")
    out.append("}\n")
    out.append("numeric\n{")
    out.append(f"   time_scheme  {cfg.get('time_scheme', 'ssprk3')}")
    out.append(f"   cfl          {cfg['cfl']!r}")
    out.append(f"   max_iter     {int(cfg.get('max_iter', 50000))}")
    out.append(f"   final_time   {cfg['final_time']!r}")
    out.append(f"   min_residue  1.0e-6")
    out.append(f"   reconstruct  {cfg.get('reconstruct', 'sp_weno')}")
    out.append(f"   net_file     {cfg.get('net_file', 'none')}")
    out.append("}\n")
    out.append("material\n{")
    if scalar:
        out.append(f"   model       {model}")
        if model == "linadv":
            v = cfg.get("vel", (1, 0, 0))
            out.append("   vel         { %r %r %r }" % tuple(float(a) for a in v))
        out.append(f"   flux        {cfg['flux']}")
    else:
        out.append(f"   gamma       {cfg.get('gamma', 1.4)!r}")
        out.append(f"   gas_const   {cfg.get('gas_const', 1.0)!r}")
        out.append("   viscosity\n   {")
        mu = cfg.get("mu_model", "constant")
        out.append(f"      model    {mu}")
        out.append(f"      mu_ref   {cfg.get('mu_ref', 0.0)!r}")
        if mu == "sutherland":
            out.append(f"      T_ref    {cfg['T_ref']!r}\n      T_0      {cfg['T_0']!r}")
        elif mu == "power":
            out.append(f"      T_ref    {cfg['T_ref']!r}\n      omega    {cfg['omega']!r}")
        out.append("   }")
        out.append(f"   prandtl     {cfg.get('prandtl', 1.0)!r}")
        out.append(f"   model       {model}")
        out.append(f"   flux        {cfg['flux']}")
        out.append(f"   EC1_fix     {cfg.get('EC1_fix', 'no')}")
    out.append("}\n")
    out.append("constants\n{")
    for k, v in cfg.get("constants", {}).items():
        out.append(f"   {k} {v!r}")
    out.append("}\n")
    out.append("initial_condition\n{")
    ic = cfg["ic"]
    if scalar:
        out.append(f"   {ic}")
    else:
        for key in ("density", "xvelocity", "yvelocity", "zvelocity", "pressure"):
            out.append(f"   {key:<12} {ic.get(key, '0.0')}")
    out.append("}\n")
    out.append("exact_soln\n{")
    ex = cfg.get("exact")
    if ex is None:
        out.append("   available   no")
    else:
        out.append("   available   yes")
        if scalar:
            out.append(f"   {ex}")
        else:
            for key in ("density", "xvelocity", "yvelocity", "zvelocity", "pressure"):
                out.append(f"   {key:<12} {ex.get(key, '0.0')}")
    out.append("}\n")
    bc = cfg.get("bc", "periodic")
    if isinstance(bc, str):
        bc = [bc] * 6
    out.append("boundary_condition\n{")
    for name, kind in zip(_BC_NAMES, bc):
        out.append(f"   {name}\n   {{\n      type {kind}\n   }}")
    out.append("}\n")
    out.append("output\n{")
    out.append(f"   OOC_study        {'yes' if cfg.get('ooc') else 'no'}")
    out.append(f"   problem_dim      {int(cfg.get('dim', 1))}")
    out.append(f"   time_stamps      {int(cfg.get('time_stamps', 1))}")
    out.append(f"   output_path      {cfg.get('output_path', '.')}")
    out.append("}\n")
    return "\n".join(out) + "\n"


def _strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    lines = []
    for line in text.splitlines():
        for mark in ("//", "#", "%"):
            p = line.find(mark)
            if p >= 0:
                line = line[:p]
        lines.append(line)
    return "\n".join(lines)


def read_param(text: str) -> dict:
    """Parse param.in text into nested dicts of raw strings.

    Sections become dicts; a line ``key value...`` becomes ``key -> 'value...'``;
    brace lists become lists of tokens.  Expressions are kept verbatim.
    """
    text = _strip_comments(text)
    toks = re.findall(r"\{|\}|[^\s{}]+(?:[ \t]+[^\s{}]+)*", text)
    pos = 0

    def parse_block():
        nonlocal pos
        d = {}
        anon = []
        while pos < len(toks):
            t = toks[pos]
            pos += 1
            if t == "}":
                if anon and not d:
                    return anon
                if anon:
                    d["_"] = anon
                return d
            if pos < len(toks) and toks[pos] == "{":
                pos += 1
                d[t.split()[0] if len(t.split()) == 1 else t] = parse_block()
            else:
                parts = t.split(None, 1)
                if len(parts) == 2:
                    if pos < len(toks) and toks[pos] == "{":
                        pos += 1
                        d[parts[0]] = parse_block()
                        continue
                    d[parts[0]] = parts[1]
                else:
                    if pos < len(toks) and toks[pos] == "{":
                        pos += 1
                        d[parts[0]] = parse_block()
                    else:
                        anon.append(parts[0])
        return d

    top = {}
    while pos < len(toks):
        name = toks[pos]
        pos += 1
        if pos < len(toks) and toks[pos] == "{":
            pos += 1
            top[name] = parse_block()
    return top
