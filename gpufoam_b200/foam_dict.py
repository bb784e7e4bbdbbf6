"""Reader (and writer) of OpenFOAM chemistry dictionaries for a RawMechanism.

The OpenFOAM side of the gpuFoam plugin builds its device mechanism from two
dictionaries: the species thermo (``physicalProperties``/``thermo.compressibleGas``:
a ``species`` list and one sub-dictionary per species with ``specie {molWeight}``
and ``thermodynamics {Tlow Thigh Tcommon highCpCoeffs lowCpCoeffs}``) and the
``reactions`` dictionary (one sub-dictionary per reaction, plus the optional
``Tlow``/``Thigh`` of all reactions). This module reads the subset of the
dictionary grammar those files use, so that real mechanisms (H2, GRI-Mech 3.0,
Yao n-dodecane in the reference's tests) run through the same loader
arithmetic, oracle and CUDA path as the synthetic ones.

Semantics restated from the reference loaders (paths relative to
gpu_chemistry/src/):

* reaction types — gpuReaction/makeGpuReactionRate.H:97-135: the type name is
  cut at the first "Reaction" substring, then one of reversibleArrhenius,
  irreversibleArrhenius, reversibleThirdBodyArrhenius,
  reversibleArrheniusLindemannFallOff, reversibleArrheniusTroeFallOff;
  anything else raises "Invalid reaction type: <name>";
* Arrhenius — :9-14 (A, beta, Ta); fall-off k0 / kInf sub-dictionaries :65-95;
  Troe F {alpha Tsss Ts Tss} :87-93;
* third-body efficiencies — :16-57: ``coeffs`` (a list of (species value)
  pairs, exactly one per species, else "Number of efficiencies is not equal to
  the number of species.") or ``defaultEfficiency`` for all species; at most
  300 species (the fixed efficiency array);
* reaction sides — the equation string is parsed as OpenFOAM's
  specieCoeffs/Reaction::setLRhs do (the plugin takes the sides of
  OpenFOAM's own reactions, makeGpuReactions.H:111-115): terms separated by
  " + ", sides by " = ", a term is an optional stoichiometric number, the
  species name and an optional "^exponent"; the exponent defaults to the
  stoichiometric coefficient; repeated species stay separate entries; species
  not in the table are dropped; more than 10 entries on a side raise "Too long
  reaction" (makeGpuReactions.H:66-68);
* reaction temperature limits — makeGpuReactions.H:117-121: ``Tlow`` default 0,
  ``Thigh`` default DBL_MAX / 10;
* species thermo — gpuThermo/makeGpuThermo.H:16-48: W = molWeight, Y = 1,
  raw NASA-7 coefficients (the x R scaling happens in the loader,
  gf_thermo_from_nasa).
"""
from __future__ import annotations

import re
from typing import Dict, List, Tuple, Union

import numpy as np

from .mechanism import (DBL_MAX_OVER_10, RATE_ARRHENIUS, RATE_LINDEMANN, RATE_THIRD_BODY, RATE_TROE,
                        RawMechanism, RawReaction)

GF_MAX_SPECIES = 300
GF_MAX_REACTION_WIDTH = 10

Value = Union[str, float, list, "FoamDict"]


class FoamDict(dict):
    """An ordered OpenFOAM dictionary: keyword -> FoamDict or a list of value tokens."""

    def sub(self, key: str) -> "FoamDict":
        v = self[key]
        if not isinstance(v, FoamDict):
            raise ValueError(f"'{key}' is not a sub-dictionary")
        return v

    def scalar(self, key: str, default=None) -> float:
        if key not in self:
            if default is None:
                raise KeyError(f"keyword '{key}' is undefined")
            return float(default)
        v = self[key]
        if isinstance(v, FoamDict) or len(v) != 1 or not isinstance(v[0], float):
            raise ValueError(f"'{key}' is not a scalar")
        return v[0]

    def word(self, key: str) -> str:
        v = self[key]
        if isinstance(v, FoamDict) or len(v) != 1 or not isinstance(v[0], str):
            raise ValueError(f"'{key}' is not a word")
        return v[0]

    def value(self, key: str) -> list:
        v = self[key]
        if isinstance(v, FoamDict):
            raise ValueError(f"'{key}' is a sub-dictionary")
        return v


class QuotedString(str):
    """A double-quoted string token (kept apart from bare words)."""


_TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<lcomment>//[^\n]*)
  | (?P<bcomment>/\*.*?\*/)
  | (?P<string>"(?:[^"\\]|\\.)*")
  | (?P<punct>[{}();])
  | (?P<atom>[^\s{}();"])
""", re.VERBOSE | re.DOTALL)

_NUMBER = re.compile(r"[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?$")


def strip_raw_string(text: str) -> str:
    """The dictionary inside a C++ raw string literal R"( ... )", if the text is one."""
    t = text.strip()
    if t.startswith('R"(') and t.endswith(')"'):
        return t[3:-2]
    return text


def _word_end(text: str, pos: int) -> int:
    """End of a bare word starting at pos: as OpenFOAM reads words, '(' and ')'
    belong to the word while they balance inside it (``CH2(S)``), so a ')' with
    no open '(' in the word ends it."""
    depth = 0
    n = len(text)
    while pos < n:
        c = text[pos]
        if c.isspace() or c in '";{}':
            break
        if c == "(":
            depth += 1
        elif c == ")":
            if depth == 0:
                break
            depth -= 1
        pos += 1
    return pos


def _tokens(text: str):
    pos = 0
    out = []
    n = len(text)
    while pos < n:
        m = _TOKEN.match(text, pos)
        if not m:
            raise ValueError(f"unreadable input at offset {pos}: {text[pos:pos + 20]!r}")
        kind = m.lastgroup
        if kind == "atom":
            end = _word_end(text, pos)
            s = text[pos:end]
            pos = end
            out.append(float(s) if _NUMBER.match(s) else s)
            continue
        pos = m.end()
        if kind in ("ws", "lcomment", "bcomment"):
            continue
        s = m.group(kind)
        if kind == "string":
            out.append(QuotedString(s[1:-1]))
        else:
            out.append(("P", s))
    return out


def _is_p(tok, c):
    return isinstance(tok, tuple) and tok[1] == c


def _parse_list(toks, i):
    """A parenthesised list starting after '(' at toks[i]; returns (list, next)."""
    out = []
    while i < len(toks):
        t = toks[i]
        if _is_p(t, ")"):
            return out, i + 1
        if _is_p(t, "("):
            sub, i = _parse_list(toks, i + 1)
            out.append(sub)
            continue
        if _is_p(t, "{") or _is_p(t, "}") or _is_p(t, ";"):
            raise ValueError(f"unexpected '{t[1]}' inside a list")
        out.append(t)
        i += 1
    raise ValueError("unterminated list")


def _parse_dict(toks, i, top):
    d = FoamDict()
    while i < len(toks):
        t = toks[i]
        if _is_p(t, "}"):
            if top:
                raise ValueError("unbalanced '}'")
            return d, i + 1
        if isinstance(t, tuple):
            raise ValueError(f"expected a keyword, found '{t[1]}'")
        key = str(t) if not isinstance(t, float) else repr(t)
        i += 1
        if i < len(toks) and _is_p(toks[i], "{"):
            sub, i = _parse_dict(toks, i + 1, False)
            d[key] = sub
            continue
        vals = []
        while i < len(toks) and not _is_p(toks[i], ";"):
            tk = toks[i]
            if _is_p(tk, "("):
                sub, i = _parse_list(toks, i + 1)
                vals.append(sub)
                continue
            if isinstance(tk, tuple):
                raise ValueError(f"unexpected '{tk[1]}' in the value of '{key}'")
            vals.append(tk)
            i += 1
        if i >= len(toks):
            raise ValueError(f"missing ';' after '{key}'")
        d[key] = vals
        i += 1
    if not top:
        raise ValueError("unterminated sub-dictionary")
    return d, i


def parse(text: str) -> FoamDict:
    """Parse OpenFOAM dictionary text (or a C++ raw string literal holding it)."""
    d, _ = _parse_dict(_tokens(strip_raw_string(text)), 0, True)
    return d


def _counted_list(v: list, what: str) -> list:
    """``N ( ... )`` or ``( ... )`` -> the list; N must match."""
    if len(v) == 2 and isinstance(v[0], float) and isinstance(v[1], list):
        if int(v[0]) != len(v[1]):
            raise ValueError(f"{what}: size {int(v[0])} but {len(v[1])} entries")
        return v[1]
    if len(v) == 1 and isinstance(v[0], list):
        return v[0]
    raise ValueError(f"{what} is not a list")


# --------------------------------------------------------------------------
# species thermo

def read_species(thermo: FoamDict) -> List[str]:
    names = _counted_list(thermo.value("species"), "species")
    if not all(isinstance(s, str) for s in names):
        raise ValueError("species must be names")
    return [str(s) for s in names]


def read_thermos(thermo: FoamDict, species: List[str]):
    n = len(species)
    W = np.empty(n)
    Tlow, Thigh, Tcommon = np.empty(n), np.empty(n), np.empty(n)
    high, low = np.empty((n, 7)), np.empty((n, 7))
    for i, s in enumerate(species):
        sd = thermo.sub(s)
        W[i] = sd.sub("specie").scalar("molWeight")
        td = sd.sub("thermodynamics")
        Tlow[i], Thigh[i], Tcommon[i] = td.scalar("Tlow"), td.scalar("Thigh"), td.scalar("Tcommon")
        for arr, key in ((high, "highCpCoeffs"), (low, "lowCpCoeffs")):
            c = _counted_list(td.value(key), key)
            if len(c) != 7 or not all(isinstance(x, float) for x in c):
                raise ValueError(f"{s}: {key} must hold 7 numbers")
            arr[i] = c
    return W, Tlow, Thigh, Tcommon, high, low


# --------------------------------------------------------------------------
# reactions

def parse_equation(eq: str, species: Dict[str, int]) -> Tuple[list, list]:
    """(lhs, rhs) lists of (index, stoich, exponent) of an equation string."""
    sides = [s.strip() for s in eq.split("=")]
    if len(sides) != 2:
        raise ValueError(f"reaction '{eq}': expected one '='")
    out = []
    for side in sides:
        terms = side.split()
        entries = []
        expect_term = True
        for t in terms:
            if t == "+":
                if expect_term:
                    raise ValueError(f"reaction '{eq}': misplaced '+'")
                expect_term = True
                continue
            if not expect_term:
                raise ValueError(f"reaction '{eq}': missing '+' before '{t}'")
            expect_term = False
            m = re.match(r"^(\d+\.?\d*|\.\d+)?(.+)$", t)
            stoich = float(m.group(1)) if m.group(1) else 1.0
            name = m.group(2)
            exponent = stoich
            if "^" in name:
                name, ex = name.split("^", 1)
                exponent = float(ex)
            if name in species:
                entries.append((species[name], stoich, exponent))
        if expect_term and terms:
            raise ValueError(f"reaction '{eq}': trailing '+'")
        if len(entries) > GF_MAX_REACTION_WIDTH:
            raise ValueError("Too long reaction")
        if not entries:
            raise ValueError(f"reaction '{eq}': a side has no known species")
        out.append(entries)
    return out[0], out[1]


def _arrhenius(d: FoamDict):
    return d.scalar("A"), d.scalar("beta"), d.scalar("Ta")


def _efficiencies(d: FoamDict, species: List[str]) -> np.ndarray:
    n = len(species)
    if n > GF_MAX_SPECIES:
        raise ValueError(f"Only up to {GF_MAX_SPECIES} species supported in ThirdBodyEfficiencies.")
    eff = np.zeros(n)
    if "coeffs" in d:
        pairs = _counted_list(d.value("coeffs"), "coeffs")
        if len(pairs) != n:
            raise ValueError("Number of efficiencies is not equal to the number of species.")
        index = {s: i for i, s in enumerate(species)}
        for p in pairs:
            if not (isinstance(p, list) and len(p) == 2 and isinstance(p[1], float)) or p[0] not in index:
                raise ValueError(f"bad third-body efficiency entry {p!r}")
            eff[index[p[0]]] = p[1]
    else:
        eff[:] = d.scalar("defaultEfficiency")
    return eff


def read_reaction(d: FoamDict, species: List[str], index: Dict[str, int]) -> RawReaction:
    t = d.word("type")
    pos = t.find("Reaction")
    tname = t[:pos] if pos >= 0 else t
    lhs, rhs = parse_equation(str(d.value("reaction")[0]), index)
    if tname in ("reversibleArrhenius", "irreversibleArrhenius"):
        A, beta, Ta = _arrhenius(d)
        return RawReaction(RATE_ARRHENIUS, tname.startswith("irr"), lhs, rhs, A=A, beta=beta, Ta=Ta)
    if tname == "reversibleThirdBodyArrhenius":
        A, beta, Ta = _arrhenius(d)
        return RawReaction(RATE_THIRD_BODY, False, lhs, rhs, A=A, beta=beta, Ta=Ta,
                           efficiencies=_efficiencies(d, species))
    if tname in ("reversibleArrheniusLindemannFallOff", "reversibleArrheniusTroeFallOff"):
        A, beta, Ta = _arrhenius(d.sub("k0"))
        Ai, bi, Ti = _arrhenius(d.sub("kInf"))
        eff = _efficiencies(d.sub("thirdBodyEfficiencies"), species)
        if tname.endswith("LindemannFallOff"):
            return RawReaction(RATE_LINDEMANN, False, lhs, rhs, A=A, beta=beta, Ta=Ta, Ainf=Ai, betainf=bi,
                               Tainf=Ti, efficiencies=eff)
        F = d.sub("F")
        troe = (F.scalar("alpha"), F.scalar("Tsss"), F.scalar("Ts"), F.scalar("Tss"))
        return RawReaction(RATE_TROE, False, lhs, rhs, A=A, beta=beta, Ta=Ta, Ainf=Ai, betainf=bi, Tainf=Ti,
                           troe=troe, efficiencies=eff)
    raise ValueError(f"Invalid reaction type: {t}")


def read_mechanism(thermo_text: str, reactions_text: str, name: str = "foam") -> RawMechanism:
    """RawMechanism of a species-thermo dictionary and a reactions dictionary."""
    thermo = parse(thermo_text)
    rdict = parse(reactions_text)
    species = read_species(thermo)
    if len(set(species)) != len(species):
        raise ValueError("duplicate species names")
    W, Tlow, Thigh, Tcommon, high, low = read_thermos(thermo, species)
    index = {s: i for i, s in enumerate(species)}
    reactions = [read_reaction(sd, species, index) for sd in rdict.sub("reactions").values()
                 if isinstance(sd, FoamDict)]
    return RawMechanism(name=name, species=species, W=W, Tlow=Tlow, Thigh=Thigh, Tcommon=Tcommon,
                        high_raw=high, low_raw=low, reactions=reactions,
                        rxn_Tlow=rdict.scalar("Tlow", 0.0), rxn_Thigh=rdict.scalar("Thigh", DBL_MAX_OVER_10))


def read_mechanism_files(thermo_path: str, reactions_path: str, name: str = None) -> RawMechanism:
    with open(thermo_path) as f:
        tt = f.read()
    with open(reactions_path) as f:
        rt = f.read()
    return read_mechanism(tt, rt, name or reactions_path)


# --------------------------------------------------------------------------
# writer: a RawMechanism as the two OpenFOAM dictionaries (the inverse of
# read_mechanism), so that seeded synthetic mechanisms can be run by an
# OpenFOAM + gpuFoam installation as they are run here

_TYPE_NAMES = {RATE_THIRD_BODY: "reversibleThirdBodyArrhenius",
               RATE_LINDEMANN: "reversibleArrheniusLindemannFallOff",
               RATE_TROE: "reversibleArrheniusTroeFallOff"}


def _num(x: float) -> str:
    """A float that reads back bit for bit (repr), without an exponent when it
    prefixes a species name."""
    return repr(float(x))


def _prefix(x: float) -> str:
    s = repr(float(x))
    if "e" in s or "E" in s or "inf" in s or "nan" in s:
        raise ValueError(f"stoichiometric coefficient {x!r} cannot be written as a prefix")
    return s[:-2] if s.endswith(".0") else s


def _side(entries, species) -> str:
    terms = []
    for i, st, ex in entries:
        t = ("" if st == 1.0 else _prefix(st)) + species[i]
        if ex != st:
            t += "^" + _num(ex)
        terms.append(t)
    return " + ".join(terms)


def _efficiencies_text(eff, species, indent) -> str:
    pad = " " * indent
    pairs = "\n".join(f"{pad}    ({s} {_num(e)})" for s, e in zip(species, eff))
    return f"{pad}coeffs {len(species)}\n{pad}(\n{pairs}\n{pad});\n"


def write_mechanism(raw: RawMechanism):
    """(thermo dictionary text, reactions dictionary text) of a RawMechanism."""
    sp = raw.species
    th = [f"species {len(sp)} ( {' '.join(sp)} );\n"]
    for i, s in enumerate(sp):
        th.append(
            f"{s}\n{{\n    specie\n    {{\n        molWeight {_num(raw.W[i])};\n    }}\n"
            f"    thermodynamics\n    {{\n        Tlow {_num(raw.Tlow[i])};\n        Thigh {_num(raw.Thigh[i])};\n"
            f"        Tcommon {_num(raw.Tcommon[i])};\n"
            f"        highCpCoeffs ( {' '.join(_num(c) for c in raw.high_raw[i])} );\n"
            f"        lowCpCoeffs ( {' '.join(_num(c) for c in raw.low_raw[i])} );\n    }}\n}}\n")
    rx = ["reactions\n{\n"]
    for k, r in enumerate(raw.reactions):
        eq = f"{_side(r.lhs, sp)} = {_side(r.rhs, sp)}"
        body = []
        if r.rate_type == RATE_ARRHENIUS:
            body.append(f"type {'irreversibleArrhenius' if r.irreversible else 'reversibleArrhenius'};")
        else:
            if r.irreversible:
                raise ValueError("the loader has no irreversible third-body or fall-off reaction type")
            body.append(f"type {_TYPE_NAMES[r.rate_type]};")
        body.append(f'reaction "{eq}";')
        lines = "".join(f"        {b}\n" for b in body)
        if r.rate_type in (RATE_ARRHENIUS, RATE_THIRD_BODY):
            lines += f"        A {_num(r.A)};\n        beta {_num(r.beta)};\n        Ta {_num(r.Ta)};\n"
            if r.rate_type == RATE_THIRD_BODY:
                lines += _efficiencies_text(r.efficiencies, sp, 8)
        else:
            lines += (f"        k0\n        {{\n            A {_num(r.A)};\n            beta {_num(r.beta)};\n"
                      f"            Ta {_num(r.Ta)};\n        }}\n"
                      f"        kInf\n        {{\n            A {_num(r.Ainf)};\n            beta {_num(r.betainf)};\n"
                      f"            Ta {_num(r.Tainf)};\n        }}\n")
            if r.rate_type == RATE_TROE:
                a, t3, t1, t2 = r.troe
                lines += (f"        F\n        {{\n            alpha {_num(a)};\n            Tsss {_num(t3)};\n"
                          f"            Ts {_num(t1)};\n            Tss {_num(t2)};\n        }}\n")
            else:
                lines += "        F\n        {\n        }\n"
            lines += "        thirdBodyEfficiencies\n        {\n" + _efficiencies_text(r.efficiencies, sp, 12) + \
                     "        }\n"
        rx.append(f"    un-named-reaction-{k}\n    {{\n{lines}    }}\n")
    rx.append("}\n")
    if raw.rxn_Tlow != 0.0:
        rx.append(f"Tlow {_num(raw.rxn_Tlow)};\n")
    if raw.rxn_Thigh != DBL_MAX_OVER_10:
        rx.append(f"Thigh {_num(raw.rxn_Thigh)};\n")
    return "".join(th), "".join(rx)


def main(argv=None) -> int:
    """python -m gpufoam_b200.foam_dict MECHANISM SEED OUTDIR: writes the seeded
    synthetic mechanism (h2_size, coverage, gri_size, large) as OUTDIR/thermo
    and OUTDIR/reactions."""
    import argparse
    import os

    from . import mechanism as M
    ap = argparse.ArgumentParser(prog="python -m gpufoam_b200.foam_dict")
    ap.add_argument("mechanism", choices=["h2_size", "coverage", "gri_size", "large"])
    ap.add_argument("seed", type=int)
    ap.add_argument("outdir")
    args = ap.parse_args(argv)
    raw = getattr(M, args.mechanism)(args.seed)
    thermo, reactions = write_mechanism(raw)
    os.makedirs(args.outdir, exist_ok=True)
    with open(os.path.join(args.outdir, "thermo"), "w") as f:
        f.write(thermo)
    with open(os.path.join(args.outdir, "reactions"), "w") as f:
        f.write(reactions)
    print(f"{args.mechanism} seed {args.seed}: {raw.n_species} species, {raw.n_reactions} reactions -> "
          f"{args.outdir}/thermo, {args.outdir}/reactions")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
