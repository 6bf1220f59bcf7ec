"""CPU tests of the command-deck subset: reading (gtcmd / splcmd rules),
the case a deck defines, and the commands it refuses."""
from __future__ import annotations

import math

import numpy as np
import pytest

from codens_b200 import cases
from codens_b200.deck import Deck, DeckError, read_commands

BOX_DECK = """\
# box, Navier-Stokes, minmod limiter
define physics gammal 1.4 pinfl 0. prandtll 0.72 prandtlt 1. &
   reyref 1.e12
define state 1 ktype 1 roi 1.2 ai 340. ti 288.15 mach 0.8 alpha -3. beta 0.
define normaliz 1
define flow equat ns3d
define numerics schema 7 muscl 1 -1. 1
create dom st 1 11 9 6
define pm_dtd ldom * lgr * eta 5.
define pm_numi ldom * lgr * kmf 1 lmax 10
define pm_dtg kdtl 1 icychr0 3 ncychro 2
create boundary st 1 1 1 1 1 1 9 1 6 i1
create boundary st 2 1 1 11 11 1 9 1 6 i2
create boundary st 3 1 1 1 11 1 1 1 6 j1
create boundary st 4 1 1 1 11 9 9 1 6 j2
create boundary st 5 1 1 1 11 1 9 1 1 k1
create boundary st 6 1 1 1 11 1 9 6 6 k2
init boundary basic 1 extr 1
init boundary basic 2 extr 1
init boundary coin 3 frc 4 kibdc 1 krr 0 ptc 1 9 1 dir +i fa +k
init boundary coin 4 frc 3 kibdc 1 krr 0 ptc 1 1 1 dir +i fa +k
init boundary coin 5 frc 6 kibdc 1 krr 0 ptc 1 1 6 dir +i +j fa
init boundary coin 6 frc 5 kibdc 1 krr 0 ptc 1 1 1 dir +i +j fa
init dom xyz * 1
init dom csvmut * 1
save dom csvmut cccc
set env_cpfw lgr * ncycle 6
compute flow
end
"""


def write_deck(tmp_path, text, name="flec"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_reading_follows_the_reference_rules():
    text = ("# a comment\n"
            "define physics gammal 1.4 &   trailing words dropped\n"
            "   pinfl 0.\r\n"
            "\n"
            "  compute   flow  \n"
            "#define numerics\n"
            "end")
    cmds = read_commands(text)
    assert [c.words for c in cmds] == [["define", "physics", "gammal", "1.4", "pinfl", "0."],
                                       ["compute", "flow"], ["end"]]
    assert [c.line for c in cmds] == [2, 5, 7]


def test_box_deck_defines_the_box_case(tmp_path):
    deck = Deck(write_deck(tmp_path, BOX_DECK))
    got = deck.case()
    want = cases.box_case((10, 8, 5), ns=True, ilim=1, skew=0.02, alpha=-3.0)
    assert [(b.ni, b.nj, b.nk) for b in got.layout.blocks] == \
        [(b.ni, b.nj, b.nk) for b in want.layout.blocks]
    assert got.layout.ld == want.layout.ld
    ga, wa = got.boundary_arrays(), want.boundary_arrays()
    for k in wa:
        assert np.array_equal(ga[k], wa[k]), k
    for f in ("gam", "pinfl", "pr", "prt", "reynz", "suth_a", "pa1", "aa1", "omg"):
        assert getattr(got.phys, f) == getattr(want.phys, f), f
    for f in ("ns", "muscl", "xk", "ilim", "eta", "kdtl", "lmax", "ischema"):
        assert getattr(got.scheme, f) == getattr(want.scheme, f), f
    assert (got.scheme.ncychro, got.scheme.icychr0) == (2, 3)
    assert deck.ncycle == 6
    assert [a[0] for a in deck.actions] == ["ingr", "infw", "svfw", "cpfw", "end"]


def test_reference_defaults(tmp_path):
    deck = Deck(write_deck(tmp_path, "create dom st 1 3 3 3\nend\n"))
    sc, ph = deck.scheme(), deck.phys()
    assert (sc.ischema, sc.muscl, sc.xk, sc.ilim, sc.eta, sc.lmax) == (1, 0, 0.0, 0, 1.0, 10)
    assert (sc.ki2, sc.ki4) == (0.0, 0.032)
    assert (sc.ncychro, sc.icychr0) == (2147483647, 10)   # dt kept after cycle 10
    assert (ph.gam, ph.pinfl, ph.pr, ph.prt) == (1.4, 1.0, 0.72, 1.0)
    assert ph.reynz == 1.7976931348623157e308
    assert deck.equat == "eu3d   "


def test_boundary_values_follow_inbdbst_and_inbdbdf(tmp_path):
    text = """define physics gammal 1.4 rgazl 287.
define state 1 roi 1.2 ti 300. mach 0.5 alpha 2. beta 1.
define normaliz 1
create dom st 1 5 4 3
create boundary st 1 1 1 1 1 1 4 1 3 i1
create boundary st 2 1 1 5 5 1 4 1 3 i2
create boundary st 3 1 1 1 5 1 1 1 3 j1
init boundary basic 1 idd 1 val/ref 1.1 1.05 2. 1.
init boundary basic 2 prd 1 state 1
init boundary basic 3 para 1
"""
    deck = Deck(write_deck(tmp_path, text))
    a, b = math.radians(2.0), math.radians(1.0)
    clmf, v = deck.bc[1]
    assert clmf == "idd " and v[:2] == [1.1, 1.05]
    np.testing.assert_allclose(v[2:], [math.cos(a) * math.cos(b), -math.cos(a) * math.sin(b),
                                       math.sin(a)], rtol=1e-15)
    gam = 1.4
    pist = 1.2 * (1.0 / gam) * 300.0
    pspi = (1.0 + 0.5 * (gam - 1.0) * 0.5 ** 2) ** (gam / (1.0 - gam))
    anz = math.sqrt(gam * 287.0 * 300.0)
    pnz = 1.2 * anz ** 2 / gam
    assert deck.bc[2][1] == [pspi * pist / pnz * (1.0 / gam)]
    assert deck.bc[3] == ("para", [])


@pytest.mark.parametrize("line,what", [
    ("init boundary basic 1 nrd 1", "boundary kind"),
    ("create boundary st 2 1 1 1 1 1 3 1 3 i1\ninit boundary basic 2 extr 1",
     "whole block faces"),
    ("define numerics fmg 1 1 0", "kfmg 0 or 3"),
    ("define pm_turbn icytur0 1", "turbulence"),
    ("frobnicate", "not handled"),
])
def test_refused_commands(tmp_path, line, what):
    base = ("create dom st 1 5 4 3\ncreate boundary st 1 1 1 1 1 1 4 1 3 i1\n"
            "init boundary basic 1 extr 1\n")
    with pytest.raises(DeckError, match=what):
        d = Deck(write_deck(tmp_path, base + line + "\n"))
        d.case()


def test_coincident_join_needs_identity_directions(tmp_path):
    text = BOX_DECK.replace("ptc 1 9 1 dir +i fa +k", "ptc 1 9 1 dir -i fa +k")
    with pytest.raises(DeckError, match="identity"):
        Deck(write_deck(tmp_path, text))


def test_per_domain_values(tmp_path):
    text = ("create dom st 1 3 3 3\ncreate dom st 2 3 3 3\n"
            "define pm_dtd ldom 1 lgr * eta 2.\ndefine pm_numd ldom 2 lgr * ki4 0.05\nend\n")
    sc = Deck(write_deck(tmp_path, text)).scheme()
    assert sc.eta_l == [2.0, 1.0] and sc.ki4_l == [0.032, 0.05] and sc.ki2_l is None
    lm = ("create dom st 1 3 3 3\ncreate dom st 2 3 3 3\n"
          "define pm_numi ldom 1 lgr * lmax 4\nend\n")
    with pytest.raises(DeckError, match="lmax differs"):
        Deck(write_deck(tmp_path, lm, "flec2")).scheme()


def test_dual_time_deck(tmp_path):
    text = BOX_DECK.replace("define numerics schema 7 muscl 1 -1. 1",
                            "define numerics schema 7 muscl 1 -1. 1 fmg 3 1 0 "
                            "dual 0 1.e-2 6 1.e-3 10")
    text = text.replace("define pm_dtg kdtl 1 icychr0 3 ncychro 2",
                        "define pm_dtg kdtl 1 icychr0 3 ncychro 2 dt1min 0.02")
    deck = Deck(write_deck(tmp_path, text))
    sc = deck.scheme()
    assert (sc.kfmg, sc.kdualns, sc.dt1min) == (3, 0, 0.02)
    assert (deck.dual_tol, deck.dual_niter) == (1.0e-2, 6)
    bad = text.replace(" dt1min 0.02", "")
    with pytest.raises(DeckError, match="physical step"):
        Deck(write_deck(tmp_path, bad, "flec2")).scheme()


@pytest.mark.parametrize("schema", [5, 9, 14])
def test_other_flux_families_from_the_deck(tmp_path, schema):
    text = BOX_DECK.replace("define numerics schema 7", f"define numerics schema {schema}")
    assert Deck(write_deck(tmp_path, text)).scheme().ischema == schema
    if schema == 5:
        eu = text.replace("define flow equat ns3d", "define flow equat eu3d")
        with pytest.raises(DeckError, match="AUSM"):
            Deck(write_deck(tmp_path, eu, "flec2")).scheme()
