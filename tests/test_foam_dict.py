"""The OpenFOAM-dictionary mechanism reader (gpufoam_b200.foam_dict), on CPU:
the dictionary grammar, equation strings, rate types, third-body efficiencies
and the loader's error behaviour; and, where the reference tree is present,
that its three test mechanisms read to exactly the mechanisms stored in the
golden fixtures (whose expected values come from the reference's own code)."""
import os

import numpy as np
import pytest

from gpufoam_b200 import foam_dict as F
from gpufoam_b200 import mechanism as M
from oracle.oracle import REFERENCE_ROOT, flatten

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
HELPERS = os.path.join(REFERENCE_ROOT, "gpu_chemistry", "unittest", "testHelpers")

THERMO = """
FoamFile { format ascii; class dictionary; }   // header, ignored
species 4 ( H2 O2 H2O CH2(S) );
/* a block
   comment */
H2  { specie { molWeight 2; }
      thermodynamics { Tlow 200; Thigh 5000; Tcommon 1000;
                       highCpCoeffs ( 3 0 0 0 0 -900 -2 ); lowCpCoeffs ( 2.3 0.008 -1.9e-05 2e-08 -7e-12 -917 0.68 ); } }
O2  { specie { molWeight 32; }
      thermodynamics { Tlow 200; Thigh 5000; Tcommon 1000;
                       highCpCoeffs ( 3.7 0.0006 -1.3e-07 1.7e-11 -9e-16 -1200 3.2 ); lowCpCoeffs ( 3.8 -0.003 9.8e-06 -9.7e-09 3.2e-12 -1000 3.7 ); } }
H2O { specie { molWeight 18; }
      thermodynamics { Tlow 200; Thigh 5000; Tcommon 1000;
                       highCpCoeffs ( 3 0.002 -6e-07 1e-10 -6e-15 -30000 5 ); lowCpCoeffs ( 4.2 -0.002 6.5e-06 -5.5e-09 1.8e-12 -30000 -0.8 ); } }
CH2(S) { specie { molWeight 14; }
      thermodynamics { Tlow 200; Thigh 5000; Tcommon 1000;
                       highCpCoeffs ( 2.3 0.004 -1.4e-06 2e-10 -1.2e-14 50000 8.6 ); lowCpCoeffs ( 4.2 -0.002 7e-06 -6e-09 1.7e-12 50000 -0.8 ); } }
"""

REACTIONS = """
reactions
{
    r0 { type reversibleArrheniusReaction; reaction "2H2 + O2 = 2H2O"; A 1e10; beta 0.5; Ta 100; }
    r1 { type irreversibleArrhenius; reaction "H2 + O2^1.5 + X = H2O + H2O^0.5"; A 2; beta 0; Ta 0; }
    r2 { type reversibleThirdBodyArrhenius; reaction "CH2(S) + H2O = CH2(S) + H2O"; A 3; beta 1; Ta 10;
         defaultEfficiency 1.5; }
    r3 { type reversibleArrheniusLindemannFallOff; reaction "H2 + H2 = H2 + H2";
         k0 { A 4; beta 0; Ta 1; } kInf { A 5; beta 0.1; Ta 2; } F { }
         thirdBodyEfficiencies { coeffs 4 ( (H2 2) (O2 1) (H2O 6) (CH2(S) 0.5) ); } }
    r4 { type reversibleArrheniusTroeFallOffReaction; reaction "O2 = O2";
         k0 { A 6; beta 0; Ta 1; } kInf { A 7; beta 0; Ta 2; } F { alpha 0.6; Tsss 100; Ts 1000; Tss 5000; }
         thirdBodyEfficiencies { coeffs ( (CH2(S) 1) (H2O 2) (O2 3) (H2 4) ); } }
}
Tlow 250;
"""


def test_grammar_and_reactions():
    raw = F.read_mechanism(THERMO, REACTIONS, "toy")
    assert raw.species == ["H2", "O2", "H2O", "CH2(S)"]
    assert list(raw.W) == [2, 32, 18, 14]
    assert raw.high_raw[3, 5] == 50000 and raw.low_raw[0, 1] == 0.008
    assert raw.rxn_Tlow == 250 and raw.rxn_Thigh == M.DBL_MAX_OVER_10
    r0, r1, r2, r3, r4 = raw.reactions
    assert (r0.rate_type, r0.irreversible, r0.A, r0.beta, r0.Ta) == (M.RATE_ARRHENIUS, False, 1e10, 0.5, 100)
    assert r0.lhs == [(0, 2.0, 2.0), (1, 1.0, 1.0)] and r0.rhs == [(2, 2.0, 2.0)]
    # exponents after '^'; unknown species dropped; repeated species kept apart
    assert r1.irreversible and r1.lhs == [(0, 1.0, 1.0), (1, 1.0, 1.5)]
    assert r1.rhs == [(2, 1.0, 1.0), (2, 1.0, 0.5)]
    assert r2.rate_type == M.RATE_THIRD_BODY and list(r2.efficiencies) == [1.5] * 4
    assert r2.lhs == [(3, 1.0, 1.0), (2, 1.0, 1.0)]
    assert r3.rate_type == M.RATE_LINDEMANN and (r3.Ainf, r3.betainf, r3.Tainf) == (5, 0.1, 2)
    assert list(r3.efficiencies) == [2, 1, 6, 0.5] and r3.lhs == [(0, 1.0, 1.0), (0, 1.0, 1.0)]
    assert r4.rate_type == M.RATE_TROE and r4.troe == (0.6, 100, 1000, 5000)
    assert list(r4.efficiencies) == [4, 3, 2, 1]


@pytest.mark.parametrize("reactions, message", [
    ('reactions { r { type reversibleArrheniusPlog; reaction "H2 = H2"; A 1; beta 0; Ta 0; } }',
     "Invalid reaction type: reversibleArrheniusPlog"),
    ('reactions { r { type reversibleThirdBodyArrhenius; reaction "H2 = H2"; A 1; beta 0; Ta 0;'
     ' coeffs 2 ( (H2 1) (O2 1) ); } }', "Number of efficiencies is not equal to the number of species."),
    ('reactions { r { type reversibleArrhenius; reaction "' + " + ".join(["H2"] * 11) + ' = H2"; A 1; beta 0;'
     ' Ta 0; } }', "Too long reaction"),
    ('reactions { r { type reversibleArrhenius; reaction "H2 + + O2 = H2"; A 1; beta 0; Ta 0; } }',
     "misplaced '+'"),
    ('reactions { r { type reversibleArrhenius; reaction "H2 + = H2"; A 1; beta 0; Ta 0; } }', "trailing '+'"),
    ('reactions { r { type reversibleArrhenius; reaction "H2 = H2"; A 1; beta 0; } }', "'Ta' is undefined"),
    ('reactions { r { type reversibleArrhenius; reaction "H2 = H2"; A 1; beta 0; Ta 0 }',
     "unexpected '}' in the value of 'Ta'"),
])
def test_errors(reactions, message):
    with pytest.raises((ValueError, KeyError), match=message.replace("(", r"\(").replace(")", r"\)")
                       .replace("+", r"\+")):
        F.read_mechanism(THERMO, reactions)


def test_species_limit():
    names = [f"S{i}" for i in range(301)]
    th = F.parse("species ( " + " ".join(names) + " );")
    species = F.read_species(th)
    d = F.parse("defaultEfficiency 1;")
    with pytest.raises(ValueError, match="Only up to 300 species"):
        F._efficiencies(d, species)


def test_counted_list_checked():
    with pytest.raises(ValueError, match="size 3 but 2"):
        F.read_species(F.parse("species 3 ( A B );"))


def test_raw_string_wrapper():
    assert F.parse('R"(a 1; b { c ( 1 2 ); })"') == {"a": [1.0], "b": {"c": [[1.0, 2.0]]}}


@pytest.mark.skipif(not os.path.isdir(HELPERS), reason="reference tree absent")
@pytest.mark.parametrize("stem", ["h2", "gri", "yao"])
def test_reference_mechanisms_match_fixtures(stem):
    raw = F.read_mechanism_files(os.path.join(HELPERS, f"{stem}_thermos.h"),
                                 os.path.join(HELPERS, f"{stem}_reactions.h"), stem)
    g = np.load(os.path.join(GOLDEN, f"foam_{stem}.npz"))
    for k, v in flatten(raw).items():
        assert np.array_equal(np.asarray(v), g[f"mech_{k}"]), k


def test_fixture_mechanism_counts():
    """Reaction-type counts of the real mechanisms as stored in the fixtures."""
    from tests.test_oracle import fixture_mech
    expect = {"foam_h2": (10, 27, {0: 18, 1: 4, 2: 4, 3: 1}),
              "foam_gri": (53, 325, {0: 284, 1: 12, 2: 3, 3: 26}),
              "foam_yao": (54, 269, {0: 238, 1: 5, 2: 1, 3: 25})}
    for name, (nS, nR, counts) in expect.items():
        raw = fixture_mech(dict(np.load(os.path.join(GOLDEN, f"{name}.npz"))))
        assert (raw.n_species, raw.n_reactions, raw.type_counts()) == (nS, nR, counts)


def test_missing_semicolon_at_end():
    with pytest.raises(ValueError, match="missing ';' after 'Tlow'"):
        F.parse("Tlow 200")


@pytest.mark.parametrize("factory, seed", [(M.h2_size, 3), (M.coverage, 4), (M.gri_size, 5), (M.large, 1)])
def test_writer_round_trip_synthetic(factory, seed):
    """write_mechanism -> read_mechanism gives back exactly the mechanism (every
    rate type, irreversible reactions, non-integer exponents, efficiencies)."""
    raw = factory(seed)
    back = F.read_mechanism(*F.write_mechanism(raw), name="back")
    assert back.species == raw.species
    for k, v in flatten(raw).items():
        assert np.array_equal(np.asarray(v), np.asarray(flatten(back)[k])), k


@pytest.mark.parametrize("name", ["foam_h2", "foam_gri", "foam_yao"])
def test_writer_round_trip_real(name):
    from tests.test_oracle import fixture_mech
    raw = fixture_mech(dict(np.load(os.path.join(GOLDEN, f"{name}.npz"))))
    back = F.read_mechanism(*F.write_mechanism(raw))
    for k, v in flatten(raw).items():
        assert np.array_equal(np.asarray(v), np.asarray(flatten(back)[k])), k


def test_writer_rejects_what_the_loader_cannot_read():
    raw = M.coverage(0)
    r = raw.reactions[[x.rate_type for x in raw.reactions].index(M.RATE_TROE)]
    r.irreversible = True
    with pytest.raises(ValueError, match="irreversible"):
        F.write_mechanism(raw)


def test_export_command(tmp_path):
    import subprocess
    import sys
    out = subprocess.run([sys.executable, "-m", "gpufoam_b200.foam_dict", "gri_size", "0", str(tmp_path)],
                         cwd=ROOT, capture_output=True, text=True, check=True, timeout=120)
    assert "53 species, 325 reactions" in out.stdout
    back = F.read_mechanism_files(str(tmp_path / "thermo"), str(tmp_path / "reactions"))
    raw = M.gri_size(0)
    for k, v in flatten(raw).items():
        assert np.array_equal(np.asarray(v), np.asarray(flatten(back)[k])), k
