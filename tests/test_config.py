"""Solver configuration parsing (CPU): the reference's JSON(C) schema
(matrix/solver/Configuration.cpp and the per-solver Configuration.cpp files),
including every configuration shipped in data/benchmarks/*.jsonc (restated
here as text fixtures in tests/golden/benchmark_configs)."""
import json
from pathlib import Path

import pytest

import graphene_b200 as gb

GOLDEN = Path(__file__).parent / "golden" / "benchmark_configs"


@pytest.mark.parametrize("path", sorted(GOLDEN.glob("*.jsonc")), ids=lambda p: p.stem)
def test_benchmark_configs_parse(path):
    text = path.read_text()
    # The solver tree is the "solver" member of the benchmark config.
    start = text.index('"solver"')
    brace = text.index("{", start)
    depth, i = 0, brace
    while True:
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                break
        i += 1
    cfg = gb.Configuration.fromJSON(text[brace:i + 1])
    assert cfg.solverName


def test_names_and_nesting():
    c = gb.Configuration.fromJSON({"type": "IterativeRefinement", "extendedPrecisionType": "float64",
                                   "innerSolver": {"type": "PBiCGStab",
                                                   "preconditioner": {"type": "ILU"}}})
    assert c.solverName == "IterativeRefinement(PBiCGStab(ILU(0)))"
    assert gb.Configuration.fromJSON({"type": "ILU", "diagonalBased": True}).solverName == "DILU"
    assert gb.Configuration.fromJSON({"type": "PBiCGStab"}).solverName == "BiCGStab"
    r = gb.Configuration.fromJSON({"type": "restarter", "maxRestarts": 3,
                                   "innerSolver": {"type": "GaussSeidel", "numSweeps": 2}})
    assert r.solverName == "Restarter of GaussSeidel"


def test_comments_and_unknown_keys():
    text = """// leading comment
    { "type": "IterativeRefinement", /* block */ "mixedPrecision": true,
      "innerSolver": {"type": "PBiCGStab", "foo": 1, "preconditioner": {"type": "ILU"}} }"""
    c = gb.Configuration.fromJSON(text)
    assert set(c.unknownKeys) == {"mixedPrecision", "foo"}


@pytest.mark.parametrize("cfg,code", [
    ({"maxIterations": 3}, 3),                                        # no type
    ({"type": "CG"}, 3),                                              # unknown solver
    ({"type": "IterativeRefinement"}, 3),                             # no innerSolver
    ({"type": "restarter"}, 3),
    ({"type": "PBiCGStab", "norm": "L3"}, 3),                         # Norm.cpp:24-35
    ({"type": "PBiCGStab", "workingType": "float16x"}, 3),            # parseType
    ({"type": "ILU", "solveMulticolor": "sometimes"}, 3),             # Configuration.cpp:66-69
    ({"type": "PBiCGStab", "maxIterations": "many"}, 3),
    ({"type": "GaussSeidel", "halo": "fresh"}, 3),                    # stale | drop
    ({"type": "ILU", "computeWarps": 3}, 1),                          # 1, 2, 4 or 8 (GR_EINVAL)
    ({"type": "ILU", "tilesPerBlock": 65}, 1),
])
def test_invalid_configs(cfg, code):
    with pytest.raises(gb.GrapheneError) as e:
        gb.Configuration.fromJSON(cfg)
    assert e.value.code == code


def test_multicolor_modes_accept_bool_and_strings():
    for v in [True, False, "on", "off", "auto", "true"]:
        gb.Configuration.fromJSON({"type": "ILU", "solveMulticolor": v, "factorizeMulticolor": v})


def test_gauss_seidel_halo_modes():
    """"halo": "stale" (the reference's sweep, halo cells hold the values of the
    last exchange) and "drop" (halo cells read as 0) are both known keys."""
    for v in ["stale", "drop"]:
        c = gb.Configuration.fromJSON({"type": "GaussSeidel", "halo": v})
        assert "halo" not in c.unknownKeys


def test_ring_kernel_options_are_known_keys():
    """The ILU ring kernel's launch options parse and are not reported as
    unknown keys."""
    c = gb.Configuration.fromJSON({"type": "ILU", "kernel": "ring", "computeWarps": 8, "tilesPerBlock": 2,
                                   "producerWarp": False, "waitingWarp": True, "pairRows": False})
    assert not set(c.unknownKeys) & {"computeWarps", "tilesPerBlock", "producerWarp", "waitingWarp", "pairRows"}
    g = gb.Configuration.fromJSON({"type": "GaussSeidel", "kernel": "wring", "pairRows": True})
    assert "pairRows" not in g.unknownKeys


def test_malformed_json():
    with pytest.raises(gb.GrapheneError) as e:
        gb.Configuration.fromJSON('{"type": "ILU",')
    assert e.value.code == 3
