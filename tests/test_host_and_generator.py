"""CPU tests of the engine's host side: the C ABI exports, host-only entry points, and the
kernel generator.  The generator test runs the emitted CUDA C statements themselves (as
text, in Python) on the CPU and compares them with the oracle for every class pair."""
import ctypes
import re
import sys
from pathlib import Path

import numpy as np
import pytest

import molints_b200 as mi

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "molecularintegrals.jl_b200"
sys.path.insert(0, str(PKG / "csrc"))
import gen_eri  # noqa: E402

sys.path.pop(0)


def _header_functions():
    text = (ROOT / "include" / "molints.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(molints_[a-z_0-9]+)\s*\(", text)))


def _header_structs():
    """{struct name: [(field, C type, array length or 0), ...]} of the typedef'd structs that
    cross the C ABI by value, read from include/molints.h."""
    text = (ROOT / "include" / "molints.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name, body in re.findall(r"typedef struct (molints_\w+) \{(.*?)\} \1;", text, flags=re.S):
        fields = []
        for decl in filter(None, (d.strip() for d in body.split(";"))):
            m = re.match(r"(?:const\s+)?(\w+)\s*(\*?)\s*(\w+)(?:\[(\d+)\])?$", " ".join(decl.split()))
            assert m, decl
            ctype = m.group(1) + ("*" if m.group(2) else "")
            fields.append((m.group(3), ctype, int(m.group(4) or 0)))
        out[name] = fields
    return out


def test_ctypes_structs_match_header():
    """The Python binding's structures have the header's fields, in order, with the same C
    types and the same size, so that every struct passed through the C ABI lines up."""
    from molints_b200 import engine
    ctype_of = {"int32_t": ctypes.c_int32, "int64_t": ctypes.c_int64, "double": ctypes.c_double}
    mirrors = {"molints_basis": engine.Basis, "molints_options": engine.Options,
               "molints_stats": engine.Stats, "molints_schedule": engine.Schedule}
    structs = _header_structs()
    assert set(mirrors) <= set(structs), sorted(structs)
    for cname, py in mirrors.items():
        want = structs[cname]
        got = py._fields_
        assert [f for f, _, _ in want] == [f for f, _ in got], cname
        for (f, ct, n), (_, pt) in zip(want, got):
            exp = ctypes.c_void_p if ct.endswith("*") else ctype_of[ct]
            if n:
                exp = exp * n
            assert ctypes.sizeof(pt) == ctypes.sizeof(exp), (cname, f)
            assert getattr(pt, "_type_", pt) == getattr(exp, "_type_", exp), (cname, f)
            if n:
                assert pt._length_ == n, (cname, f)


def test_julia_shim_structs_match_header():
    """The Julia ccall shim of INTEGRATION.md declares MolintsBasis and MolintsOptions with the
    header's fields, in order, with matching types (isbits structs pass by Ref as the C structs)."""
    text = (ROOT / "INTEGRATION.md").read_text()
    jl = {"Int32": "int32_t", "Int64": "int64_t", "Float64": "double"}
    structs = _header_structs()
    for jname, cname in (("MolintsBasis", "molints_basis"), ("MolintsOptions", "molints_options")):
        body = re.search(r"struct %s\n(.*?)\nend" % jname, text, flags=re.S).group(1)
        body = re.sub(r"#[^\n]*", "", body)
        fields = re.findall(r"(\w+)::(Ptr\{\w+\}|\w+)", body)
        want = structs[cname]
        assert [f for f, _ in fields] == [f for f, _, _ in want], jname
        for (f, jt), (_, ct, _) in zip(fields, want):
            assert (jt.startswith("Ptr{") and ct.endswith("*")) or jl.get(jt) == ct, (jname, f, jt, ct)


@pytest.fixture(scope="module")
def lib():
    from molints_b200 import engine
    return engine.load_library()


def test_library_exports_every_header_symbol(lib):
    from molints_b200 import engine
    declared = _header_functions()
    assert declared, "no functions found in include/molints.h"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(engine.EXPORTED_SYMBOLS) == declared


def test_host_only_entry_points(lib):
    from molints_b200 import engine
    assert lib.molints_abi_version() == 1
    for n in (0, 1, 2, 16, 104, 330):
        assert lib.molints_npacked(n) == n * (n + 1) * (n * n + n + 2) // 8
    assert lib.molints_npacked(-1) == -1
    sh = mi.config2()
    arrs = engine._BasisArrays(sh)
    assert lib.molints_nbf(ctypes.byref(arrs.c)) == 60
    o = engine.Options()
    lib.molints_default_options(ctypes.byref(o))
    assert (o.method, o.precision, o.boys, o.fp32_cutoff, o.screen_cutoff) == (0, 0, 0, 0.0, 0.0)


def test_create_without_device_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = ctypes.c_void_p()
    rc = lib.molints_create(ctypes.byref(h), 0, 0, 0)
    assert rc == -4 and not h.value


def test_null_arguments_rejected(lib):
    assert lib.molints_create(None, 0, 0, 0) == -1
    assert lib.molints_eri_packed(None, None, None, None, 0, None) == -1
    assert lib.molints_plan_execute(None, None) == -1
    assert lib.molints_destroy(None) == 0


# ------------------------------------------------------------------ generator
def _py_statement(line: str) -> str:
    line = line.strip().rstrip(";")
    line = re.sub(r"^const (VT|double) ", "", line)
    return line.replace("(VT)", "").replace("(double)", "")


def _emulate_class(X, Y, bra_prims, ket_prims, A, B, C, D):
    """Run the generator's VRR/HRR statements for one quartet; return res[] (normalised)."""
    (la, lb), (lc, ld) = X, Y
    e, f = la + lb, lc + ld
    entries = gen_eri.vrr_entries(la, e, lc, f)
    hp = gen_eri.HrrPlan(la, lb, lc, ld)
    acc = [0.0] * (len(hp.acc_a) * len(hp.acc_c))
    env = {"acc": acc}
    for (a, ca), (b, cb) in bra_prims:
        for (c, cc), (d, cd) in ket_prims:
            z, et = a + b, c + d
            P = (a * A + b * B) / z
            Q = (c * C + d * D) / et
            r2 = 1.0 / (z + et)
            PQ = P - Q
            T = z * et * r2 * PQ @ PQ
            kab = ca * cb * np.exp(-a * b / z * np.sum((A - B) ** 2)) / z
            kcd = cc * cd * np.exp(-c * d / et * np.sum((C - D) ** 2)) / et
            pref = 2 * np.pi ** 2.5 * kab * kcd * np.sqrt(r2)
            from oracle import oracle as o
            with o.exact_boys():
                F = o.farray(e + f + 1, T)
            env.update(pref=pref, F=F, oo2z=0.5 / z, oo2e=0.5 / et, oo2ze=0.5 * r2,
                       rho_z=et * r2, rho_e=z * r2)
            for i, x in enumerate("xyz"):
                env["PA" + x] = P[i] - A[i]
                env["QC" + x] = Q[i] - C[i]
                env["WP" + x] = -et * r2 * PQ[i]
                env["WQ" + x] = z * r2 * PQ[i]
            for k in entries:
                exec(_py_statement(gen_eri.vrr_line(*k)), {}, env)
            for a_ in hp.acc_a:
                for c_ in hp.acc_c:
                    acc[hp.acc_index[(a_, c_)]] += env[gen_eri.vname(a_, c_, 0)]
    for i, x in enumerate("xyz"):
        env["AB" + x] = (A - B)[i]
        env["CD" + x] = (C - D)[i]
    for ln in hp.lines:
        exec(_py_statement(ln), {}, env)
    res = []
    for a, b, c, d, expr in hp.targets:
        g = gen_eri.comp_norm(a) * gen_eri.comp_norm(b) * gen_eri.comp_norm(c) * gen_eri.comp_norm(d)
        res.append(eval(expr, {}, env) * g)
    return np.array(res)


def _norm_prims(l, prims):
    ex = np.array([p[0] for p in prims])
    co = np.array([p[1] for p in prims])
    s = sum(co[i] * co[j] * (2 * np.sqrt(ex[i] * ex[j]) / (ex[i] + ex[j])) ** (l + 1.5)
            for i in range(len(ex)) for j in range(len(ex)))
    cn = 1 / np.sqrt(s)
    return [(e, c * cn * (2 * e / np.pi) ** 0.75 * (4 * e) ** (l / 2)) for e, c in zip(ex, co)]


@pytest.mark.parametrize("X,Y", gen_eri.class_pairs())
def test_generated_statements_match_oracle(oracle, X, Y):
    rng = np.random.default_rng(hash((X, Y)) % 2**32)
    centres = [rng.uniform(-1.2, 1.2, 3) for _ in range(4)]
    ls = [X[0], X[1], Y[0], Y[1]]
    shells = []
    for l, xyz in zip(ls, centres):
        k = int(rng.integers(1, 3))
        shells.append((xyz, l, mi.basis._random_shell(rng, l, k, 0.3, 6.0)))
    sh = mi.Shells.from_list(shells)
    with oracle.exact_boys():
        ref = oracle.shell_quartet(sh, 0, 1, 2, 3).reshape(-1)
    bra = [(p, q) for p in _norm_prims(ls[0], shells[0][2]) for q in _norm_prims(ls[1], shells[1][2])]
    ket = [(p, q) for p in _norm_prims(ls[2], shells[2][2]) for q in _norm_prims(ls[3], shells[3][2])]
    got = _emulate_class(X, Y, bra, ket, *[np.asarray(c) for c in centres])
    assert np.max(np.abs(got - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_generator_sources_are_current():
    """The committed generated/ kernels are exactly what gen_eri.py emits."""
    for X, Y in gen_eri.class_pairs():
        p = gen_eri.OUT_DIR / f"eri_{gen_eri.tag_of(X, Y)}.cu"
        assert p.read_text() == gen_eri.emit_class_pair(X, Y), p.name
    assert (gen_eri.HERE / "eri_dispatch.h").read_text() == gen_eri.emit_dispatch(gen_eri.class_pairs())
