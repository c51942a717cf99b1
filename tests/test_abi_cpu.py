"""The C ABI library: it loads without a GPU, exports what include/ltlgpu.h declares,
and its host-only pieces (Scarlet reader, status strings) behave as the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

from ltlb200 import api, gen
from helpers import fixture_path, load_fixture

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ltlgpu.h")).read()
    return sorted(set(re.findall(r"LTLG_API\s+[\w\s\*]+?\b(ltlg_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(api.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(api.EXPORTED)


def test_abi_version_and_status_strings():
    lib = api.lib()
    assert lib.ltlg_abi_version() == api.ABI_VERSION
    assert api.status_string(api.NOT_FOUND) == "not_found"
    assert api.status_string(api.INPUT_LIMITS) == "see_the_error"


def test_scarlet_reader_matches_python_reader():
    for name in ("ham1_len3.trace", "f10x10_p3_s0.trace", "cfg1_deep.trace", "len64.trace"):
        a = api.read_scarlet(fixture_path(name))
        b = load_fixture(name)
        assert a.num_pos == b.num_pos and a.num_neg == b.num_neg and a.alphabet == b.alphabet
        assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.steps, b.steps)


def test_scarlet_reader_rules(tmp_path):
    # file order of the letters maps values; the letter index is the sorted order;
    # a trailing newline on the letter line is ignored; other characters advance the index
    p = tmp_path / "t.trace"
    p.write_text("1,0;0,1\n1,1\n---\n0,0;1 ,0\n---\nops\n---\nq,p\n")
    t = api.read_scarlet(str(p))
    assert t.alphabet == "pq" and t.num_pos == 2 and t.num_neg == 1
    q, pp = 1 << (ord("q") - 97), 1 << (ord("p") - 97)
    assert list(t.steps) == [q, pp, q | pp, 0, q]  # "1 ,0": '1' is index 0 (q), ' ' advances
    assert list(t.offsets) == [0, 2, 3, 5]
    u = gen.from_scarlet_text(p.read_text())
    assert np.array_equal(u.steps, t.steps) and u.alphabet == t.alphabet


def test_generator_is_deterministic():
    a = gen.generate(5, 3, 50, 50, 4, 20, 0.5, 6)
    b = gen.generate(5, 3, 50, 50, 4, 20, 0.5, 6)
    assert np.array_equal(a.steps, b.steps) and a.hidden == b.hidden
    h = gen.generate_hamming(3, 4, 40, 40, 20, 48, 0.5, 5)
    assert h.num_pos == 40 and h.num_neg == 40
    # every negative differs from every positive
    lines = h.trace_lines()
    assert not set(lines[:40]) & set(lines[40:])


def test_hamming_negatives_are_near_misses():
    """Each negative is a positive with 1-3 bits flipped, falsifies the hidden formula, and
    repeats no positive."""
    h = gen.generate_hamming(7, 4, 60, 60, 20, 48, 0.5, 6)
    offs, steps = h.offsets, h.steps
    tr = [steps[offs[i]:offs[i + 1]] for i in range(h.n)]
    pos, neg = tr[:60], tr[60:]
    for t in neg:
        best = min((sum(bin(int(a) ^ int(b)).count("1") for a, b in zip(t, p)) for p in pos if len(p) == len(t)),
                   default=None)
        assert best is not None and 1 <= best <= 3
    cs = h.atom_cs()
    assert cs.shape[0] == 4


def test_one_shot_learn_checks_limits_before_the_device():
    """ltlg_learn refuses traces longer than 63 steps before it looks for a device, as the
    reference checks its limits before its first device call (ltli6463.cu:1078-1083)."""
    res = api.learn(load_fixture("len64.trace"), costs=(2, 1, 1, 1, 1, 1, 1, 1))
    assert res.status == api.INPUT_LIMITS and res.formula == "see_the_error" and res.cost == 2
    over = load_fixture("over64.trace")
    assert api.learn(over, limit_traces=True).status == api.INPUT_LIMITS


def test_scarlet_reader_fuzz(tmp_path):
    """The library's one-pass reader and the Python restatement agree on malformed files:
    stray characters, carriage returns, empty lines, values beyond the alphabet, missing or
    extra separators, no final newline."""
    rng = np.random.default_rng(7)
    parts = ["0", "1", "1", ",", ";", " ", "\r", "x", "\n"]
    for case in range(300):
        lines = []
        for _ in range(int(rng.integers(0, 12))):
            if rng.random() < 0.15:
                lines.append("---")
            else:
                lines.append("".join(rng.choice(parts[:-1]) for _ in range(int(rng.integers(0, 14)))))
        letters = "".join(rng.choice(list("abcdpqrz,; \r")) for _ in range(int(rng.integers(0, 8))))
        text = "\n".join(lines + [letters]) + ("\n" if rng.random() < 0.5 else "")
        p = tmp_path / f"f{case}.trace"
        p.write_bytes(text.encode())
        a = api.read_scarlet(str(p))
        b = gen.from_scarlet_text(text)
        assert (a.num_pos, a.num_neg, a.alphabet) == (b.num_pos, b.num_neg, b.alphabet), (case, text)
        assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.steps, b.steps), (case, text)


def test_scarlet_reader_large_file(tmp_path):
    """A file of 50,000 + 50,000 traces of 10 steps over 4 letters (the shape of the
    reference's largest Varying_size inputs) reads in well under a second."""
    import time
    rng = np.random.default_rng(1)
    vals = rng.integers(0, 4, size=(100000, 10))
    onehot = ["1,0,0,0", "0,1,0,0", "0,0,1,0", "0,0,0,1"]
    lines = [";".join(onehot[v] for v in row) for row in vals]
    text = "\n".join(lines[:50000] + ["---"] + lines[50000:] + ["---", "G,F,!,U,&,|,X", "---", "a,b,c,d"])
    p = tmp_path / "nw50000.trace"
    p.write_text(text)
    t0 = time.perf_counter()
    t = api.read_scarlet(str(p))
    el = time.perf_counter() - t0
    assert t.num_pos == 50000 and t.num_neg == 50000 and t.alphabet == "abcd"
    assert np.array_equal(t.steps, (1 << vals.ravel()).astype(np.uint32))
    assert el < 1.0, el


def test_scarlet_writer_round_trip(tmp_path):
    """Instance.to_scarlet (the layout of code/dc.py:8-21) read back by the library."""
    for seed in range(4):
        inst = gen.generate(seed, 3, 30, 25, 1, 20, 0.5, 5)
        p = tmp_path / f"r{seed}.trace"
        p.write_text(inst.to_scarlet())
        t = api.read_scarlet(str(p))
        assert (t.num_pos, t.num_neg, t.alphabet) == (inst.num_pos, inst.num_neg, inst.alphabet)
        assert np.array_equal(t.offsets, inst.offsets) and np.array_equal(t.steps, inst.steps)


def _raw(alphabet="pq", offsets=(0, 2, 3), steps=(1, 2, 3)):
    return gen.Instance(1, 1, alphabet, np.array(steps, dtype=np.uint32), np.array(offsets, dtype=np.int32))


def test_malformed_traces_are_refused_before_the_device():
    """Decreasing or negative offsets and letters outside a-z would become negative shift
    counts; every entry point that reads traces refuses them with LTLG_BAD_ARGS before it
    looks for a device."""
    good = _raw()
    bad = [_raw(offsets=(0, 3, 2)), _raw(offsets=(-1, 1, 2)), _raw(alphabet="pQ"), _raw(alphabet="p1")]
    L = api.lib()
    f = L.ltlg_learn_noalloc
    f.argtypes = [ctypes.POINTER(api.Traces), ctypes.POINTER(api.Options), ctypes.c_char_p, ctypes.c_int32,
                  ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64)]
    f.restype = ctypes.c_int
    for inst in bad:
        r = api.learn(inst)
        assert r.status == api.BAD_ARGS and r.formula == "bad_arguments"
        with pytest.raises(ValueError, match="bad_arguments"):
            api.evaluate(inst, "p")
        t, keep = api._traces(inst)
        o = api.make_options()
        buf = ctypes.create_string_buffer(64)
        assert f(ctypes.byref(t), ctypes.byref(o), buf, 64, None, None) == api.BAD_ARGS
    # a well-formed set gets past the checks to the device lookup
    assert api.learn(good).status != api.BAD_ARGS


def test_generate_many_in_child_interpreters_equals_sequential():
    """The parallel generator (child interpreters, chunks of specs) gives the sequential
    instances, in order."""
    from ltlb200 import workloads
    specs = list(workloads.cfg4_specs(10, seed=3))
    par = list(workloads.generate_many("generate", specs, workers=3, chunk=4))
    seq = [gen.generate(*s) for s in specs]
    assert len(par) == len(seq) == 10
    for a, b in zip(par, seq):
        assert (a.num_pos, a.num_neg, a.alphabet, a.hidden) == (b.num_pos, b.num_neg, b.alphabet, b.hidden)
        assert np.array_equal(a.steps, b.steps) and np.array_equal(a.offsets, b.offsets)


def test_header_is_plain_c(tmp_path):
    """include/ltlgpu.h compiles as C99 (-pedantic, warnings as errors) and a C program links
    against the library and calls it: the boundary needs no C++ on the caller's side."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "c_abi.c"
    src.write_text('#include "ltlgpu.h"\n'
                   "int main(void) { ltlg_options o; ltlg_default_options(&o);\n"
                   "  return (o.max_cost == 500 && ltlg_abi_version() == LTLG_ABI_VERSION) ? 0 : 1; }\n")
    lib_dir = os.path.dirname(api.LIB_PATH)
    exe = tmp_path / "c_abi"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", lib_dir, "-lltlgpu", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)]).returncode == 0


def test_struct_layouts_match_ctypes(tmp_path):
    """Sizes and field offsets of the ABI structs as a C compiler lays them out equal the ctypes
    mirrors the Python binding passes across the boundary."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    checks = {"ltlg_engine_config": (api.EngineConfig, ["slots_log2", "cache_bytes", "small_rows", "wait_spins",
                                                        "small_level"]),
              "ltlg_options": (api.Options, ["max_cost", "stop_at_found", "time_limit_s"]),
              "ltlg_result": (api.Result, ["formula", "levels", "blocks", "launches"]),
              "ltlg_traces": (api.Traces, ["alphabet", "steps", "offsets"]),
              "ltlg_block_record": (api.BlockRecord, ["candidates", "features"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ltlgpu.h"', "int main(void) {"]
    for cname, (_, fields) in checks.items():
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {f}));')
    lines.append("  return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for _, (cls, fields) in checks.items():
        want.append(ctypes.sizeof(cls))
        want.extend(getattr(cls, f).offset for f in fields)
    assert got == want


def test_null_handles_and_no_device():
    """Accessors and destructors accept null handles; creating an engine or a batch on a host
    without a CUDA device returns LTLG_NO_DEVICE and no handle (no CPU fallback)."""
    if _has_cuda():
        pytest.skip("checks the no-device path")
    L = api.lib()
    assert L.ltlg_engine_stream(None) is None and L.ltlg_batch_stream(None, 0) is None
    L.ltlg_engine_destroy(None)
    L.ltlg_batch_destroy(None)
    L.ltlg_result_free(None)
    L.ltlg_traces_free(None)
    cfg = api.EngineConfig()
    L.ltlg_default_engine_config(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    assert L.ltlg_engine_create(ctypes.byref(cfg), ctypes.byref(h)) == api.NO_DEVICE and not h.value
    assert L.ltlg_batch_create(ctypes.byref(cfg), 2, ctypes.byref(h)) == api.NO_DEVICE and not h.value


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
