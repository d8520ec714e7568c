"""The C-ABI library loads and exports every symbol include/lj_gpu.h declares (no GPU calls)."""

import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(lj_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("lj_gpu_create", "lj_gpu_step", "lj_gpu_compute_forces", "lj_gpu_debug_pairs",
                 "lj_gpu_debug_cells", "lj_gpu_rdf", "lj_initial_condition"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from lennardjonesium import _native
    L = _native.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
        assert name in _native.SIGNATURES, name


def test_status_strings_and_default_params():
    from lennardjonesium import _native
    L = _native.lib()
    assert L.lj_gpu_status_string(0) == b"ok"
    assert L.lj_gpu_status_string(5) == b"neighbour list capacity exceeded"
    p = _native.Params()
    L.lj_gpu_default_params(ctypes.byref(p))
    assert p.cutoff_distance == 2.5 and p.time_delta == 0.005 and p.periodic == 1


def test_create_rejects_bad_arguments():
    """Argument checks run on the host before any device call."""
    from lennardjonesium import _native
    L = _native.lib()
    p = _native.Params()
    L.lj_gpu_default_params(ctypes.byref(p))
    ctx = ctypes.c_void_p()
    p.particle_count = 0
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG
    p.particle_count = 1 << 26  # past the 26-bit slot field of a neighbour entry
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG
    p.particle_count = 10
    for k in range(3):
        p.box[k] = 2.0  # box below the cutoff (particle_pair_filter.cpp:61-64)
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG
    for k in range(3):
        p.box[k] = 10.0
    p.cutoff_distance = 1.0  # rc^2 <= 2^(1/3) (lennard_jones_force.cpp:45)
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG
    p.cutoff_distance = 2.5
    p.periodic = 0  # forces without the periodic boundary are not a reference configuration
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG
    p.periodic = 1
    p.mixed_per_pair = 2  # a flag: 0 or 1
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG
    p.mixed_per_pair, p.force_block = 0, 96  # block sizes 64, 128, 256
    assert L.lj_gpu_create(ctypes.byref(p), ctypes.byref(ctx)) == _native.LJ_ERR_ARG


def test_host_initial_condition_matches_oracle():
    """The library's InitialCondition equals the oracle's (same seed contract)."""
    import ljref
    from lennardjonesium import initial_condition
    for N, T, rho, seed in [(500, 0.5, 0.8, 117208264), (864, 0.722, 0.8442, 5489), (100, 0.6, 1.0, 17)]:
        x, v, L = initial_condition(N, T, rho, seed)
        xo, vo, Lo = ljref.initial_state(N, T, rho, seed)
        assert L == Lo
        assert np.array_equal(x, xo)
        assert np.allclose(v, vo, rtol=0, atol=1e-14)


def _header_struct(name):
    """(type, field) pairs of `typedef struct name {...} name;` in include/lj_gpu.h, in order."""
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "lj_gpu.h").read_text(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"(const char\*|unsigned long long|long long|double|int|unsigned)\s*(.*)", decl)
        assert m, decl
        for field in m.group(2).split(","):
            out.append((m.group(1), field.strip()))
    return out


_CTYPES = {"int": ctypes.c_int, "double": ctypes.c_double, "long long": ctypes.c_longlong,
           "unsigned": ctypes.c_uint, "const char*": ctypes.c_char_p}


@pytest.mark.parametrize("name,cls", [("lj_params", "Params"), ("lj_stats", "Stats"), ("lj_thermo", "Thermo"),
                                      ("lj_phase_times", "PhaseTimes"), ("lj_sim_config", "SimConfig"),
                                      ("lj_sim_result", "SimResult"), ("lj_batch_system", "BatchSystem"),
                                      ("lj_adj_params", "AdjParams"), ("lj_observation", "Observation"),
                                      ("lj_batch_tuning", "BatchTuning")])
def test_ctypes_structs_follow_the_header(name, cls):
    """The Python binding's structs list the header's fields in the header's order and types."""
    from lennardjonesium import _native
    fields = getattr(_native, cls)._fields_
    decl = _header_struct(name)
    assert len(fields) == len(decl)
    for (fname, ftype), (ctype, cdecl) in zip(fields, decl):
        m = re.match(r"(\w+)(?:\[(\d+)\])?$", cdecl)
        assert fname == m.group(1)
        base = _CTYPES[ctype]
        assert ftype == (base * int(m.group(2)) if m.group(2) else base)


def _pxd_struct(name):
    """(type, field) lines of `ctypedef struct name:` in include/lj_gpu.pxd, in order."""
    text = (ROOT / "include" / "lj_gpu.pxd").read_text()
    block = re.search(r"ctypedef struct %s:\n((?:        .*\n)+)" % name, text).group(1)
    return [" ".join(line.split()) for line in block.splitlines()]


@pytest.mark.parametrize("name", ["lj_params", "lj_thermo"])
def test_cython_declarations_follow_the_header(name):
    """The Cython declarations a maintainer cimports list the header's fields in order and type."""
    assert _pxd_struct(name) == [f"{t} {f}" for t, f in _header_struct(name)]


def test_cython_functions_follow_the_header():
    """Every function include/lj_gpu.pxd declares has the header's parameter and return types."""
    text = (ROOT / "include" / "lj_gpu.pxd").read_text()
    protos = _prototypes()
    found = 0
    for m in re.finditer(r"^    ([\w \*]+?)\b(lj_\w+)\(([^)]*)\)", text, flags=re.M):
        ret, name, params = " ".join(m.group(1).split()), m.group(2), m.group(3)
        want_ret, want_params = protos[name]
        assert ret.replace(" *", "*") == want_ret.replace(" *", "*"), name
        got = [" ".join(p.split()).replace(" *", "*") for p in params.split(",") if p.strip()]
        want = [re.sub(r"\s*\b\w+$", "", p).replace(" *", "*") for p in want_params]
        assert got == want, (name, got, want)
        found += 1
    assert found >= 10


def _prototypes():
    """name -> (return type, [parameter types]) of the functions include/lj_gpu.h declares."""
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "lj_gpu.h").read_text(), flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(lj_\w+)\s*\(([^)]*)\)\s*;", text):
        ret = " ".join(m.group(1).split())
        params = [" ".join(p.split()) for p in m.group(3).split(",") if p.strip() and p.strip() != "void"]
        out[m.group(2)] = (ret, params)
    return out


def _kind(decl):
    """ctypes class a C parameter or return type maps to (pointers as c_void_p)."""
    decl = re.sub(r"\b(const|struct)\b", "", decl)
    if "*" in decl:
        return "char_p" if re.match(r"\s*char\s*\*\s*\w*$", decl) else "ptr"
    words = decl.split()
    base = " ".join(w for w in words[:-1]) if len(words) > 1 else words[0]
    return {"int": "int", "double": "double", "long long": "longlong", "void": "void",
            "unsigned": "uint", "unsigned long long": "ulonglong"}[base]


def test_signatures_follow_the_header():
    """Return and parameter types of every binding agree with the header's prototypes."""
    from lennardjonesium import _native
    as_kind = {None: "void", ctypes.c_int: "int", ctypes.c_double: "double", ctypes.c_longlong: "longlong",
               ctypes.c_uint: "uint", ctypes.c_ulonglong: "ulonglong", ctypes.c_char_p: "char_p",
               ctypes.c_void_p: "ptr"}
    protos = _prototypes()
    for name, (res, args) in _native.SIGNATURES.items():
        ret, params = protos[name]
        want_ret = "ptr" if "*" in ret else _kind(ret + " x")
        if want_ret == "ptr" and res is ctypes.c_char_p:
            want_ret = "char_p"
        assert as_kind[res] == want_ret, name
        assert len(args) == len(params), name
        for a, prm in zip(args, params):
            k = _kind(prm)
            assert as_kind[a] == k or (k == "char_p" and as_kind[a] == "ptr"), (name, prm)


def test_window_stats_host_matches_the_analyzer_formulas():
    """lj_window_stats_host restates physics/analyzers.cpp:44-159 over records
    (no GPU): numpy's two-pass statistics agree to 1e-12."""
    from lennardjonesium import _native
    rng = np.random.default_rng(7)
    n, N, rho = 300, 4000, 0.8
    rec = np.zeros((n, 7))
    rec[:, 0] = 0.005 * np.arange(1, n + 1)
    rec[:, 5] = 1.2 + 0.01 * rng.standard_normal(n)
    rec[:, 3] = -4000 + rng.standard_normal(n)
    rec[:, 4] = 2000 + 10 * rng.standard_normal(n)
    rec[:, 6] = 0.3 * rec[:, 0] + 1e-3 * rng.standard_normal(n)
    o = _native.Observation()
    assert _native.lib().lj_window_stats_host(rec.ctypes.data_as(ctypes.c_void_p), n, N, rho, ctypes.byref(o)) == 0
    T = rec[:, 5].mean()
    varT = rec[:, 5].var(ddof=1)
    want = [T, rho, rec[:, 3].mean(), rho * (T + rec[:, 4].mean() / (3 * N)),
            1.5 / (1 - 1.5 * N * varT / T ** 2), np.cov(rec[:, 0], rec[:, 6])[0, 1] / rec[:, 0].var(ddof=1) / 6]
    got = [getattr(o, f) for f, _ in o._fields_]
    assert np.allclose(got, want, rtol=1e-12, atol=0)
    # the package's wrapper returns the same fields by name
    from lennardjonesium import window_stats_host
    assert list(window_stats_host(rec, N, rho).values()) == got
