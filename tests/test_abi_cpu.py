"""C-ABI checks that need no GPU: the library loads, exports every declared symbol, and its host-side
logic (seed split, host RNG, comb, exchange plan) agrees with the oracle."""
import os
import re

import numpy as np
import pytest

from oracle import afqmc as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(afqmc_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(capi_lib):
    decl = _declared_functions()
    assert len(decl) > 30
    missing = [n for n in decl if not hasattr(capi_lib, n)]
    assert not missing, missing


def test_binding_covers_header(capi_lib):
    from safire_b200 import capi
    assert set(_declared_functions()) <= set(capi.exported_symbols())


def test_status_strings(capi_lib):
    assert capi_lib.afqmc_status_string(0) == b"ok"
    assert capi_lib.afqmc_status_string(2) == b"shape mismatch"


def test_split_seed_matches_oracle(capi_lib):
    from safire_b200 import afqmc as A
    for seed, rank, stream in [(0, 0, 0), (0, 0, 1), (12345, 3, 1), (-7, 200, 255)]:
        assert A.split_seed(seed, rank, stream) == O.split_seed(seed, rank, stream)


def test_host_rng_matches_oracle(capi_lib):
    from safire_b200 import afqmc as A
    s = O.split_seed(5, 1, 0)
    a = A.HostRandomGenerator(s).sample_uniform(3000)
    b = O.HostRandomGenerator(s).sample_uniform(3000)
    assert np.array_equal(a, b)


def test_comb_bit_exact(capi_lib):
    from safire_b200 import afqmc as A
    rs = np.random.default_rng(11)
    for trial in range(20):
        n = int(rs.integers(1, 300))
        w = rs.random(n) * rs.choice([0.0, 1.0, 3.0], size=n, p=[0.1, 0.6, 0.3])
        if w.sum() <= 1e-6:
            w[0] = 1.0
        s = O.split_seed(trial, 0, 0)
        a = A.comb(A.HostRandomGenerator(s), w, n)
        b = O.comb(O.HostRandomGenerator(s), w, n)
        assert np.array_equal(a, b)


def test_comb_collapse_status(capi_lib):
    from safire_b200 import afqmc as A
    from safire_b200.capi import AfqmcError
    with pytest.raises(AfqmcError) as e:
        A.comb(A.HostRandomGenerator(1), np.zeros(4), 4)
    assert e.value.status == 8


def test_plan_walker_exchange_matches_oracle(capi_lib):
    from safire_b200 import afqmc as A
    rs = np.random.default_rng(3)
    for _ in range(40):
        nr = int(rs.integers(1, 7))
        counts = [int(c) for c in rs.integers(1, 12, size=nr)]
        ntot = sum(counts)
        off = np.zeros(ntot, dtype=np.int32)
        for _k in range(ntot):
            off[rs.integers(0, ntot)] += 1
        assert A.plan_walker_exchange(off, counts) == O.plan_walker_exchange(off, counts)


def test_plan_rejects_non_conserving_offspring(capi_lib):
    from safire_b200 import afqmc as A
    from safire_b200.capi import AfqmcError
    with pytest.raises(AfqmcError):
        A.plan_walker_exchange([2, 0, 0], [3])


def test_cpp_consumer(tmp_path):
    """A C++ program built against include/afqmc_c.h and the shared library alone (what a SAFIRE
    build links): its host-side results equal the oracle's."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    lib = os.path.join(ROOT, "safire_b200", "_lib")
    exe = tmp_path / "abi_consumer"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "abi_consumer.cpp"), "-L", lib,
                    "-lsafire_afqmc", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    lines = dict(line.split(" ", 1) for line in out.strip().splitlines())
    assert int(lines["seed"]) == O.split_seed(7, 1, 0)
    w = np.array([0.5, 1.5, 0.25, 2.0, 0.75, 1.0])
    off = O.comb(O.HostRandomGenerator(O.split_seed(3, 0, 0)), w, w.size)
    assert [int(x) for x in lines["offspring"].split()] == list(off)
    plan = O.plan_walker_exchange(off, [3, 3])
    p = [int(x) for x in lines["plan"].split()]
    assert p[0] == len(plan) and p[1:] == [int(v) for e in plan for v in e]
    # reference {0,1,2}: {3,1,2} single, {0,2,4} single with an odd column order, {5,4,1} double
    assert lines["excitations"].split() == ["4", "0:+1", "1:+1", "2:-1", "3:+1"]
    assert lines["status"] == "invalid argument"
