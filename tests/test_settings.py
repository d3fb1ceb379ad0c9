"""CPU checks of the .PUR settings parser and the tPurificationSet mirror.

The parser restates initialize_purification (source/purification_settings.f90:
91-218) on the tokens of readline (source/readline.f90:1-64, checktype in
source/readl2.f90:52-90); the defaults are those of the derived types
(source/purification_settings.f90:29-86).  The C library's
ptbgpu_default_settings is host code and is compared here without a GPU.
"""
import ctypes

import pytest

from ptb_b200 import api
from ptb_b200 import settings as ps
from ptb_b200.settings import PurificationSettings, PurSettingsError


def test_defaults_are_the_derived_type_defaults():
    s = PurificationSettings()
    assert (s.mode, s.type, s.cycles, s.prlvl) == (ps.FULL, ps.SIGN_DIAGONALIZATION, 40, 1)
    assert (s.dev, s.check) == (True, False)
    assert (s.submatrix_mode, s.submatrix_columns) == (ps.SUBMATRIX_SYGV, ps.ATOMS_COLUMNS)
    assert (s.metric_type, s.metric_cycles, s.metric_iterative) == (ps.INV_SQRT, 50, False)
    assert (s.chempot_cycles, s.chempot_guess, s.chempot_increment) == (60, -1.5, 0.1)


def test_c_library_defaults_match_the_mirror():
    lib = api.load_library()
    c = api._Settings()
    lib.ptbgpu_default_settings(ctypes.byref(c))
    py = PurificationSettings().to_c(api._Settings)
    for name, _ in api._Settings._fields_:
        assert getattr(c, name) == getattr(py, name), name


def test_code_values_match_the_header():
    # source/purification_settings.f90:6-27 and include/ptbgpu.h
    assert (ps.FULL, ps.SUBMATRIX) == (1, 2)
    assert (ps.SINGLE_COLUMNS, ps.ATOMS_COLUMNS, ps.FULL_MATRIX, ps.KMEANS_R_HEURISTIC) == (1, 2, 3, 4)
    assert (ps.SUBMATRIX_SIGN, ps.SUBMATRIX_SYGV) == (1, 2)
    assert (ps.MCWEENY, ps.SIGN_ITER_PADE, ps.SIGN_ITER_NEWTON, ps.SIGN_DIAGONALIZATION) == (1, 2, 3, 4)
    assert (ps.INV, ps.INV_SQRT, ps.SQRT_) == (1, 2, 3)


def test_submatrix_run_file():
    # the layout of the per-run settings files: mode, a bare flag, the submatrix keys,
    # and commented-out alternatives
    text = ("submatrix_columns = kmeans_r_heuristic\n"
            "!submatrix_columns = full_matrix\n"
            "submatrix_mode = submatrix_sygv\n"
            "mode = submatrix\n"
            "check\n")
    s = PurificationSettings().read(text)
    assert s.mode == ps.SUBMATRIX
    assert s.submatrix_columns == ps.KMEANS_R_HEURISTIC
    assert s.submatrix_mode == ps.SUBMATRIX_SYGV
    assert s.check and s.dev


@pytest.mark.parametrize("key,value,field,code", [
    ("mode", "full", "mode", ps.FULL),
    ("mode", "submatrix", "mode", ps.SUBMATRIX),
    ("submatrix_columns", "single_columns", "submatrix_columns", ps.SINGLE_COLUMNS),
    ("submatrix_columns", "atoms_columns", "submatrix_columns", ps.ATOMS_COLUMNS),
    ("submatrix_columns", "full_matrix", "submatrix_columns", ps.FULL_MATRIX),
    ("submatrix_columns", "kmeans_r_heuristic", "submatrix_columns", ps.KMEANS_R_HEURISTIC),
    ("submatrix_mode", "submatrix_sign", "submatrix_mode", ps.SUBMATRIX_SIGN),
    ("submatrix_mode", "submatrix_sygv", "submatrix_mode", ps.SUBMATRIX_SYGV),
    ("type", "mcweeny", "type", ps.MCWEENY),
    ("type", "pade", "type", ps.SIGN_ITER_PADE),
    ("type", "newton", "type", ps.SIGN_ITER_NEWTON),
    ("type", "diag", "type", ps.SIGN_DIAGONALIZATION),
    ("metric", "inverse", "metric_type", ps.INV),
    ("metric", "inverse_sqrt", "metric_type", ps.INV_SQRT),
    ("metric", "sqrt", "metric_type", ps.SQRT_),
])
def test_every_keyword(key, value, field, code):
    s = PurificationSettings().read(f"{key} = {value}\n")
    assert getattr(s, field) == code


@pytest.mark.parametrize("key,msg", [
    ("mode", "Error: .PUR contains invalid type definition"),
    ("submatrix_columns", "Error: .PUR contains invalid type definition"),
    ("submatrix_mode", "Error: .PUR contains invalid type definition"),
    ("type", "Error: .PUR contains invalid type definition"),
    ("metric", "Error: .PUR contains invalid metric definition."),
])
def test_invalid_values_stop_with_the_reference_message(key, msg):
    with pytest.raises(PurSettingsError) as ei:
        PurificationSettings().read(f"{key} = nonsense\n")
    assert str(ei.value) == msg
    # a number is not a string token, so the third string is empty: also invalid
    with pytest.raises(PurSettingsError):
        PurificationSettings().read(f"{key} = 2\n")


def test_numeric_keys_truncate_like_int():
    s = PurificationSettings().read("cycles = 77.9\nchempot_cycles = 12\npr = 2\nchempot_increment = 0.5\n")
    assert (s.cycles, s.chempot_cycles, s.prlvl) == (77, 12, 2)
    # chempot%increment = int(floats(1)): a fractional increment becomes 0
    assert s.chempot_increment == 0.0
    s = PurificationSettings().read("chempot_increment = 3.7\n")
    assert s.chempot_increment == 3.0


def test_numeric_key_without_a_number_keeps_the_default():
    s = PurificationSettings().read("cycles = many\npr =\n")
    assert (s.cycles, s.prlvl) == (40, 1)
    # nan / inf are not numbers here (the reference's int() of them is undefined)
    s = PurificationSettings().read("cycles = nan\nchempot_cycles = inf\npr = -inf\n")
    assert (s.cycles, s.chempot_cycles, s.prlvl) == (40, 60, 1)


def test_integer_settings_out_of_range_raise_the_settings_error():
    for line in ("cycles = 1e30", "pr = -1e19", "chempot_increment = 9.3e18"):
        with pytest.raises(PurSettingsError):
            PurificationSettings().read(line)


def test_strings_and_numbers_are_counted_apart():
    # readline numbers string and numeric tokens separately: a number before the
    # '=' still counts as the value, and the '=' is still the second string
    s = PurificationSettings().read("cycles 25 =\n")
    assert s.cycles == 25
    s = PurificationSettings().read("cycles\t=\t30\n")
    assert s.cycles == 30


def test_bare_flags_and_comments():
    s = PurificationSettings().read("! comment = with equals\niterative_inversion\ncheck\ndev\n\n   \n")
    assert s.metric_iterative and s.check and s.dev
    # a flag written as a key/value pair is not a flag
    s = PurificationSettings().read("check = 1\n")
    assert not s.check
    # true/false are logical tokens, never strings
    s = PurificationSettings().read("true\n")
    assert s == PurificationSettings()


def test_unknown_keys_are_ignored():
    s = PurificationSettings().read("filter = 1e-5\ncolor = blue\nsomething\n")
    assert s == PurificationSettings()


def test_line_is_read_into_80_characters():
    # "cycles =" is 8 characters: with 72 blanks the value starts in column 81
    # and is lost, so cycles keeps its default; with 70 it ends in column 80
    s = PurificationSettings().read("cycles =" + " " * 72 + "55\n")
    assert s.cycles == 40
    s = PurificationSettings().read("cycles =" + " " * 70 + "55\n")
    assert s.cycles == 55


def test_later_lines_override_earlier_ones(tmp_path):
    f = tmp_path / ".PUR"
    f.write_text("type = pade\ncycles = 10\ntype = newton\n")
    s = PurificationSettings.from_file(f)
    assert s.type == ps.SIGN_ITER_NEWTON and s.cycles == 10


def test_to_c_carries_every_field():
    s = PurificationSettings(mode=2, type=3, cycles=11, prlvl=0, nel=64, submatrix_mode=1, submatrix_columns=4,
                             metric_type=1, metric_cycles=7, metric_iterative=True, chempot_cycles=9,
                             chempot_guess=-0.25, chempot_increment=2.0)
    c = s.to_c(api._Settings)
    assert [getattr(c, f) for f, _ in api._Settings._fields_] == [2, 3, 11, 0, 64, 1, 4, 1, 7, 1, 9, -0.25, 2.0]


def test_arbitrary_lines_parse_or_raise_the_settings_error():
    """Any text made of the parser's keywords, values, numbers and junk either
    parses or raises PurSettingsError (the reference's error stop), nothing else."""
    from hypothesis import given, settings as hsettings, strategies as st

    words = st.sampled_from(["mode", "type", "metric", "cycles", "pr", "chempot_cycles", "chempot_increment",
                             "submatrix_mode", "submatrix_columns", "=", "!", "!x", "full", "submatrix", "pade",
                             "newton", "diag", "mcweeny", "inverse", "sqrt", "inverse_sqrt", "single_columns",
                             "kmeans_r_heuristic", "submatrix_sygv", "check", "dev", "iterative_inversion", "true",
                             "false", "1", "2.5", "-3", "1e-5", "1d-3", "nan", "inf", "x=y", "", "\t"])
    line = st.lists(words, max_size=6).map(" ".join)
    text = st.lists(line, max_size=8).map("\n".join)

    @hsettings(max_examples=300, deadline=None)
    @given(text)
    def check(t):
        try:
            s = PurificationSettings().read(t)
        except PurSettingsError:
            return
        assert s.mode in (ps.FULL, ps.SUBMATRIX) and 1 <= s.type <= 4 and 1 <= s.metric_type <= 3

    check()


def test_print_settings_layout_and_mode_line_quirk():
    thr = float(__import__("numpy").float32(1e-4))   # thrs%normal for 2000 <= ndim < 15000
    s = PurificationSettings(type=ps.MCWEENY, mode=ps.SUBMATRIX)
    lines = s.format_settings(thr).splitlines()
    assert lines[0] == "" and lines[1] == "*" * 72 and lines[2] == "*" * 26 + " PURIFICATION MODE " + "*" * 27
    # the mode line selects on the type: McWeeny (1) prints 'Full matrix' although mode is submatrix
    assert lines[6] == "  Calculation mode :            " + " " * 6 + "Full matrix"
    assert lines[7] == "  Purification type:            " + " " * 6 + "McWeeny Grand Canonical Purification"
    assert lines[8] == "  Iteration Cycles:           " + " " * 8 + "40"
    text = s.format_settings(thr)
    # (2x,a,3x,f13.8) and (2x,a,3x,e13.6) after the reference's padded labels
    assert "\n  Initial Chemical Potential:   " + " " * 3 + "  -1.50000000\n" in text
    assert "\n  Threshold:                      " + " " * 3 + " 0.100000E-03\n" in text
    assert text.endswith("\n" + "*" * 72 + "\n\n")
    # Newton (3): no mode text, so the open record continues with the type label
    t = PurificationSettings(type=ps.SIGN_ITER_NEWTON).format_settings(thr).splitlines()
    assert t[6] == ("  Calculation mode :            " + " " * 6 + "  Purification type:            " + " " * 6
                    + "Iterative Sign: Newton-Schulz")
    # print level 0: no metric, chempot or threshold blocks
    q = PurificationSettings(prlvl=0).format_settings(thr)
    assert "__metric__" not in q and "Threshold" not in q and "Print Level:" in q


def test_fortran_e_format():
    from ptb_b200.settings import _fortran_e
    assert _fortran_e(9.999999747378752e-05, 13, 6) == " 0.100000E-03"
    assert _fortran_e(1e-3, 13, 6) == " 0.100000E-02"
    assert _fortran_e(-123.456, 13, 6) == "-0.123456E+03"
    assert _fortran_e(0.0, 13, 6) == " 0.000000E+00"
