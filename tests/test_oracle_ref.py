"""The oracle against the reference (CPU only).

Pins the CPU restatement (oracle/fs_oracle.cpp), driven through the product's
own parser, network builder and output writers, to the output files the
reference compiled from its sources wrote for the same .conf/.pro
(tests/golden, made by tests/golden/make_golden.py): every file must be
byte-identical.
"""
import os

import pytest

from conftest import golden_cases, model_for, compare_outputs, first_diff, generated_case, GOLDEN


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_files(built, oracle, case, tmp_path):
    fb = built
    m = model_for(fb, case)
    ctx = oracle.oracle_create(m.desc())
    try:
        m.run_with(oracle.oracle_engine(), ctx, str(tmp_path))
    finally:
        oracle.oracle_destroy(ctx)
    bad = compare_outputs(case, str(tmp_path))
    msgs = [(f, first_diff(os.path.join(GOLDEN, case, f), os.path.join(str(tmp_path), f))) for f in bad]
    assert not bad, msgs


def test_oracle_matches_reference_at_connectome_scale(built, oracle, tmp_path):
    # the 20,000-neuron connectome-shaped network with delays 0 (about 4.1 M
    # synapse entries on the reference's single-target path,
    # code/EqsGnl2.cpp:404-502), 100 ms, reference run with -t 1: the
    # oracle's Spikes.dat and rate file equal the reference's (size, SHA-256)
    case = "connectome20k_d0"
    generated_case(case, tmp_path)
    m = model_for(built, case, conf_dir=tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    ctx = oracle.oracle_create(m.desc())
    try:
        m.run_with(oracle.oracle_engine(), ctx, str(out))
    finally:
        oracle.oracle_destroy(ctx)
    assert not compare_outputs(case, str(out))


def test_golden_cases_cover_the_features():
    # spike, rate, sum-rate, receptor currents, dV overflow, gating variables,
    # membrane potential, aligned spikes, repeats
    names = set()
    for c in golden_cases():
        names.update(os.listdir(os.path.join(GOLDEN, c)))
    for f in ("Spikes.dat", "FR.dat", "FRs.dat", "Isyn.dat", "ov.dat", "gv.dat", "Mem.dat", "sa.dat", "Spikes.dat_3"):
        assert f in names
    spikes = sum(1 for _ in open(os.path.join(GOLDEN, "two_pop", "Spikes.dat")))
    assert spikes > 1000  # a busy raster, not a silent network
