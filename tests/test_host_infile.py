"""The C++ host's input-file parser (include/dq_host.h) without a GPU.

Line by line it is checked against the reference's own stringSplit and
stringTrim (cppUtility.cpp:82-106), compiled from the reference's source into
oracle/_ref when that source is present; whole files against the key semantics
of systemClass::parseInFile (systemClass.cu:184-735), on the reference's own
example input file when it is present and on files written here.
"""
import os

import pytest

from dynaquant_b200 import _lib
from dynaquant_b200 import host

REF_INFILE = "/root/reference/infile.in"

TRICKY_LINES = [
    "dt              = 1.0",
    "writebinarypops\t\t=\t0",
    "printallpops        =   1   !Write out all populations",
    "sigmastatdis    =   300     !in wavenumbers",
    "! simtype         = SIM_TYPE_CONST_HAM",
    "! Only lines with '=' are considered",
    "outfolder = outDataFolder",
    "hamfile = data-example/hamInner.dat",
    "key =  \t value with tab",
    "key=value",
    "key =x",
    "key = ",
    "   spaced key   =   spaced value   ",
    "\tm\t= \t12\t",
    "a = b = c",
    "no assignment here",
    "",
    "x =",
]


def _ref_lines_available():
    from oracle import oracle as O
    O.build()
    return os.path.exists(O.REF_INFILE)


@pytest.mark.skipif(not os.path.exists("/root/reference/cppUtility.cpp"), reason="reference sources absent")
def test_line_split_matches_the_reference_functions():
    from oracle import oracle as O
    assert _ref_lines_available()
    lines = list(TRICKY_LINES)
    if os.path.exists(REF_INFILE):
        lines += open(REF_INFILE).read().splitlines()
    for ln in lines:
        ref = O.ref_parse_line(ln)
        got = host.split_line(ln)
        if ref == "throws":
            # the one deviation: the reference's substr throws on a line ending in '='
            assert got is not None and got[1] == "", ln
        else:
            assert got == ref, (ln, got, ref)


@pytest.mark.skipif(not os.path.exists(REF_INFILE), reason="reference example input absent")
def test_reference_example_infile_parses_to_its_values():
    d = host.parse_infile(REF_INFILE)
    assert d["dt"] == 1.0 and d["totalsteps"] == 400 and d["ensembleruns"] == 5 and d["m"] == 12
    assert d["ensembleavgmode"] == _lib.ENS_AVG_FIRST and d["ka_substeps"] == 5
    assert d["absorbspec"] == 0 and d["cdspec"] == 0 and d["lineshapedress"] == 0 and d["gausswidth"] == 1000.0
    assert d["dostatelooping"] == 1 and d["stepsperloop"] == 200
    assert d["writeoutpops"] == 1 and d["printallpops"] == 1 and d["writebinarypops"] == 0
    assert d["printpop"] == [300, 301, 359] + [-1] * 7
    assert d["print_partic"] == 0 and d["writeoutstates"] == 0
    assert d["initstate"] == 300 and d["initfromfile"] == 0
    assert d["initstatefile"] == "data-example/sample_multisite_init.dat"
    assert d["propmode"] == _lib.PROP_LANCZOS and d["simtype"] == _lib.SIM_ZZ_REAL_NOISE
    assert d["staticdis"] == 1 and d["sigmastatdis"] == 300.0 and d["temperature"] == 77.0
    assert d["zz_specd_file"] == "data-example/specd_tresp.dat"
    assert d["hamfile"] == "data-example/hamInner.dat" and d["dipolefile"] == "data-example/dips_1roll.dat"
    assert d["outfolder"] == "outDataFolder" and d["debug_diags"] == 0
    assert d["n_unknown"] == 0


def _write(tmp_path, text, name="in.in"):
    p = tmp_path / name
    p.write_text(text)
    return p


def test_defaults_are_the_references():
    d = host.defaults()
    assert d["simtype"] == _lib.SIM_CONST_HAM and d["propmode"] == _lib.PROP_LANCZOS
    assert d["ensembleavgmode"] == _lib.ENS_AVG_NONE and d["temperature"] == -1.0
    assert d["tk_p"] == 10 and d["tk_m_aux"] == 24 and d["outfolder"] == "outFolderDefault"
    assert d["printpop"] == [-1] * 10 and d["precision"] == _lib.PREC_FP64 and d["pop_every"] == 1


def test_own_file_every_key(tmp_path):
    p = _write(tmp_path, "\n".join([
        "! a comment line = with an equals sign",
        "dt = 0.5",
        "totalsteps = 64",
        "ensembleavgmode = ENS_AVG_MODE_CONTINUATION",
        "ensembleruns = 16",
        "m = 20",
        "ka_substeps = 3",
        "simtype = SIM_TYPE_KUBO_ANDERSON",
        "propmode = PROP_MODE_TAYLOR_LANCZOS",
        "tk_p = 4",
        "tk_m_aux = 12",
        "tkmatfile = b.dat",
        "staticdis = 1",
        "sigmastatdis = 150.5  ! cm^-1",
        "ka_paramsfile = ka.dat",
        "hsr_stddevfile = hsr.dat",
        "temperature = 300",
        "absorbspec = 1",
        "lineshapedress = 1",
        "gausswidth = 250",
        "dipolefile = d.dat",
        "posfile = r.dat",
        "writeoutstates = 8",
        "print_partic = 1",
        "initfromfile = 1",
        "initstatefile = s.dat",
        "printpop4 = 17",
        "precision = PREC_MIXED",
        "seed = 12345678901",
        "pop_every = 4",
        "unknown_key = 3",
        "hamfile\t=\th.dat",
    ]) + "\n")
    d = host.parse_infile(p)
    assert d["dt"] == 0.5 and d["totalsteps"] == 64 and d["ensembleavgmode"] == _lib.ENS_AVG_CONTINUATION
    assert d["ensembleruns"] == 16 and d["m"] == 20 and d["ka_substeps"] == 3
    assert d["simtype"] == _lib.SIM_KUBO_ANDERSON and d["propmode"] == _lib.PROP_TAYLOR_LANCZOS
    assert d["tk_p"] == 4 and d["tk_m_aux"] == 12 and d["tkmatfile"] == "b.dat"
    assert d["staticdis"] == 1 and d["sigmastatdis"] == 150.5 and d["temperature"] == 300.0
    assert d["ka_paramsfile"] == "ka.dat" and d["hsr_stddevfile"] == "hsr.dat"
    assert d["absorbspec"] == 1 and d["lineshapedress"] == 1 and d["gausswidth"] == 250.0
    assert d["dipolefile"] == "d.dat" and d["posfile"] == "r.dat"
    assert d["writeoutstates"] == 8 and d["print_partic"] == 1
    assert d["initfromfile"] == 1 and d["initstatefile"] == "s.dat"
    assert d["printpop"][4] == 17 and d["printpop"][0] == -1
    assert d["precision"] == _lib.PREC_MIXED and d["seed"] == 12345678901 and d["pop_every"] == 4
    assert d["hamfile"] == "h.dat"
    assert d["n_unknown"] == 1


@pytest.mark.parametrize("line", ["writeoutpops = 2", "staticdis = -1", "print_partic = 5",
                                  "simtype = SIM_TYPE_SOMETHING", "propmode = PROP_MODE_X"])
def test_invalid_values_abort_as_the_reference_does(tmp_path, line):
    p = _write(tmp_path, f"dt = 1.0\n{line}\n")
    with pytest.raises(_lib.DQError) as e:
        host.parse_infile(p)
    assert e.value.code == _lib.DQ_ERR_ARG


def test_absorb_and_cd_together_abort(tmp_path):
    p = _write(tmp_path, "absorbspec = 1\ncdspec = 1\n")
    with pytest.raises(_lib.DQError):
        host.parse_infile(p)


def test_unknown_average_mode_falls_back_to_none(tmp_path):
    p = _write(tmp_path, "ensembleavgmode = ENS_AVG_MODE_WHATEVER\n")
    assert host.parse_infile(p)["ensembleavgmode"] == _lib.ENS_AVG_NONE


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(_lib.DQError):
        host.parse_infile(tmp_path / "absent.in")


def test_run_refuses_incomplete_input_without_touching_a_gpu(tmp_path):
    """A missing hamfile is refused before any device call."""
    p = _write(tmp_path, "dt = 1.0\ntotalsteps = 4\n")
    with pytest.raises(_lib.DQError) as e:
        host.run_infile(p, base_dir=tmp_path)
    assert e.value.code == _lib.DQ_ERR_ARG
    p = _write(tmp_path, "dt = 1.0\ntotalsteps = 4\nhamfile = nothere.dat\n")
    with pytest.raises(_lib.DQError) as e:
        host.run_infile(p, base_dir=tmp_path)
    assert "failed to open" in str(e.value)
