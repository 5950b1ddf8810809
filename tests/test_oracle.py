"""The oracle pinned against the reference (CPU only).

* golden fixtures (tests/golden, generated from the reference's own engine by
  tests/golden/make_golden.py): the oracle's parser reproduces the
  reference's PT lists and the oracle's serial engine reproduces the
  reference's FP64 t_CPU states bit for bit;
* closed forms (H benchmark, Grover, QFT) agree with the fixtures;
* when oracle/_ref is built in this container, random circuits run through
  the reference and through the oracle agree bit for bit.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import circuit_lang as cl
from oracle import closed_forms as cf
from oracle import cpu
from simulador_quantico_b200 import workloads as wl

GOLDEN = sorted((Path(__file__).resolve().parent / "golden").glob("*.npz"))
SPECS = None


def golden_specs():
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", Path(__file__).parent / "golden" / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return dict(mod.cases())


@pytest.fixture(scope="module")
def specs():
    return golden_specs()


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 40


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_parser_matches_reference_pts(path, specs):
    g = np.load(path)
    spec = specs[path.stem]
    c = spec.build(cl.Circuit())
    t, cm, cv, m = c.as_arrays()
    assert np.array_equal(t, g["target"])
    assert np.array_equal(cm, g["cmask"])
    assert np.array_equal(cv, g["cval"])
    assert np.abs(m - g["matrix"]).max(initial=0.0) < 1e-15


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_serial_bit_exact_vs_reference(path):
    g = np.load(path)
    n = int(g["qubits"])
    ops = (g["target"], g["cmask"], g["cval"], g["matrix"])
    s = cpu.run_serial(cpu.basis_state(n, int(g["init_index"])), n, ops, prec="f64")
    assert np.array_equal(s, g["state_f64"])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_regions_vs_reference_fp32(path):
    g = np.load(path)
    n = int(g["qubits"])
    ops = (g["target"], g["cmask"], g["cval"], g["matrix"])
    s = cpu.run_regions(cpu.basis_state(n, int(g["init_index"]), np.complex64), n, ops, prec="f32", threads=4)
    assert np.abs(s - g["state_f32_par"]).max() < 2e-6


def test_closed_forms_vs_fixtures():
    d = Path(__file__).resolve().parent / "golden"
    for n in (10, 14):
        g = np.load(d / f"hadamard_{n}.npz")
        assert np.abs(g["state_f64"] - cf.hadamard_all(n)).max() < 1e-14
        # tests/smoke_test.sh:70-76 prints amplitude 0 with %.6f
        assert f"{g['state_f64'][0].real:.6f}" == f"{2.0 ** (-n / 2):.6f}"
    g = np.load(d / "grover_ref_9.npz")
    k = wl.grover_reference_iterations(9)
    assert np.abs(g["state_f64"] - cf.grover_reference_form(9, 42, k)).max() < 1e-13
    g = np.load(d / "qft_8.npz")
    assert np.abs(g["state_f64"] - cf.qft_basis(8, 77)).max() < 1e-14
    g = np.load(d / "grover_search_9.npz")
    k = wl.grover_search(9, 300).meta["iterations"]
    assert np.abs(g["state_f64"] - cf.grover_search(9, 300, k)).max() < 1e-13


def test_serial_and_regions_agree():
    n = 12
    spec = wl.random_layered(n, 3, seed=4)
    ops = spec.build(cl.Circuit()).as_arrays()
    a = cpu.run_serial(cpu.basis_state(n, 0), n, ops)
    b = cpu.run_regions(cpu.basis_state(n, 0), n, ops, threads=4, coalesced_bits=3, region_bits=6)
    assert np.abs(a - b).max() < 1e-14


@pytest.mark.skipif(not cpu.ref_available("f64"), reason="reference not built in this container")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_vs_live_reference(seed):
    from tests.helpers import random_gate_circuit_spec

    n = 9
    spec = random_gate_circuit_spec(n, 60, seed)
    init = np.random.default_rng(seed).standard_normal(1 << n) + 0j
    r = cpu.RefDGM(n, "f64")
    for name, m in spec.gates.items():
        r.add_gate(name, m)
    r.set_state(init)
    for steps, it, reset in spec.calls:
        r.set_function(steps, it, reset)
    t, cm, cv, m = r.pts()
    r.tuning(cpu.RefDGM.T_CPU)
    r.execute(1)
    ref_serial = r.state()
    r.set_state(init)
    r.tuning(cpu.RefDGM.T_PAR_CPU, thread_count=4, cpu_region_bits=6, cpu_coalesced_bits=3)
    r.execute(1)
    ref_par = r.state()
    r.close()
    ops = (t, cm, cv, m)
    assert np.array_equal(cpu.run_serial(init, n, ops), ref_serial)
    assert np.array_equal(cpu.run_regions(init, n, ops, threads=4, coalesced_bits=3, region_bits=6), ref_par)
