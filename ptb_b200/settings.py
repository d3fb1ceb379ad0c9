"""tPurificationSet mirror and the .PUR settings parser.

Follows source/purification_settings.f90:6-218: the same mode codes and
defaults, the same ``key = value`` / bare-flag grammar, the same errors on
invalid values, and the same quirk that ``chempot_increment`` is truncated by
``int()`` (source/purification_settings.f90:193-195).  format_settings
restates print_settings (source/purification_settings.f90:222-300).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

FULL, SUBMATRIX = 1, 2
SINGLE_COLUMNS, ATOMS_COLUMNS, FULL_MATRIX, KMEANS_R_HEURISTIC = 1, 2, 3, 4
SUBMATRIX_SIGN, SUBMATRIX_SYGV = 1, 2
MCWEENY, SIGN_ITER_PADE, SIGN_ITER_NEWTON, SIGN_DIAGONALIZATION = 1, 2, 3, 4
INV, INV_SQRT, SQRT_ = 1, 2, 3

_MODE = {"full": FULL, "submatrix": SUBMATRIX}
_COLUMNS = {"single_columns": SINGLE_COLUMNS, "atoms_columns": ATOMS_COLUMNS,
            "full_matrix": FULL_MATRIX, "kmeans_r_heuristic": KMEANS_R_HEURISTIC}
_SMMODE = {"submatrix_sign": SUBMATRIX_SIGN, "submatrix_sygv": SUBMATRIX_SYGV}
_TYPE = {"mcweeny": MCWEENY, "pade": SIGN_ITER_PADE, "newton": SIGN_ITER_NEWTON,
         "diag": SIGN_DIAGONALIZATION}
_METRIC = {"inverse": INV, "inverse_sqrt": INV_SQRT, "sqrt": SQRT_}


class PurSettingsError(ValueError):
    pass


@dataclass
class PurificationSettings:
    mode: int = FULL
    type: int = SIGN_DIAGONALIZATION
    cycles: int = 40
    prlvl: int = 1
    dev: bool = True
    check: bool = False
    nel: int = 0
    submatrix_mode: int = SUBMATRIX_SYGV
    submatrix_columns: int = ATOMS_COLUMNS
    metric_type: int = INV_SQRT
    metric_cycles: int = 50
    metric_iterative: bool = False
    chempot_cycles: int = 60
    chempot_guess: float = -1.5
    chempot_increment: float = 0.1

    def to_c(self, struct_type):
        return struct_type(self.mode, self.type, self.cycles, self.prlvl, self.nel, self.submatrix_mode,
                           self.submatrix_columns, self.metric_type, self.metric_cycles,
                           int(self.metric_iterative), self.chempot_cycles, self.chempot_guess,
                           self.chempot_increment)

    # initialize_purification, source/purification_settings.f90:91-218
    def read(self, text: str) -> "PurificationSettings":
        for raw in text.splitlines():
            strs, floats = _readline(raw)
            if not strs and not floats:
                continue
            arg1 = strs[0] if strs else ""
            if arg1.startswith("!"):
                continue
            arg2 = strs[1] if len(strs) > 1 else ""
            if arg2 == "=":
                arg3 = strs[2] if len(strs) > 2 else ""
                num = floats[0] if floats else None
                if arg1 == "mode":
                    self.mode = _pick(_MODE, arg3, "Error: .PUR contains invalid type definition")
                elif arg1 == "submatrix_columns":
                    self.submatrix_columns = _pick(_COLUMNS, arg3, "Error: .PUR contains invalid type definition")
                elif arg1 == "submatrix_mode":
                    self.submatrix_mode = _pick(_SMMODE, arg3, "Error: .PUR contains invalid type definition")
                elif arg1 == "type":
                    self.type = _pick(_TYPE, arg3, "Error: .PUR contains invalid type definition")
                elif arg1 == "metric":
                    self.metric_type = _pick(_METRIC, arg3, "Error: .PUR contains invalid metric definition.")
                elif arg1 == "cycles" and num is not None:
                    self.cycles = _int_value(num)
                elif arg1 == "chempot_cycles" and num is not None:
                    self.chempot_cycles = _int_value(num)
                elif arg1 == "chempot_increment" and num is not None:
                    self.chempot_increment = float(_int_value(num))
                elif arg1 == "pr" and num is not None:
                    self.prlvl = _int_value(num)
            else:
                if arg1 == "dev":
                    self.dev = True
                elif arg1 == "check":
                    self.check = True
                elif arg1 == "iterative_inversion":
                    self.metric_iterative = True
        return self

    # print_settings, source/purification_settings.f90:222-300
    def format_settings(self, thrs_normal: float) -> str:
        """The settings block the reference prints, edit descriptor by edit
        descriptor.  Its quirk is kept: the 'Calculation mode' line selects on
        the solver type, not on the mode (type 1 prints 'Full matrix', type 2
        'Submatrix method', types 3 and 4 nothing), and because that line is a
        non-advancing write, an unmatched case leaves the record open so that
        the 'Purification type' label continues on the same line."""
        out = ["", "*" * 72, "*" * 26 + " PURIFICATION MODE " + "*" * 27, "*" * 72,
               "  __SETTINGS__", "  __general__"]
        rec = "  Calculation mode :            " + " " * 6          # (2x,a,6x), advance='no'
        mode_text = {FULL: "Full matrix", SUBMATRIX: "Submatrix method"}.get(self.type)
        if mode_text is not None:
            out.append(rec + mode_text)
            rec = ""
        rec += "  Purification type:            " + " " * 6         # (2x,a,6x), advance='no'
        cycles = "  Iteration Cycles:           " + " " * 8 + str(self.cycles)
        type_text = {MCWEENY: "McWeeny Grand Canonical Purification", SIGN_ITER_PADE: "Iterative Sign: Pade",
                     SIGN_DIAGONALIZATION: "Sign Diagonalization",
                     SIGN_ITER_NEWTON: "Iterative Sign: Newton-Schulz"}.get(self.type)
        if type_text is not None:
            out.append(rec + type_text)
            rec = ""
            if self.type != SIGN_DIAGONALIZATION and self.prlvl > 0:
                out.append(cycles)
        lead = rec   # an open record (no type matched) is continued by the next write
        if self.prlvl > 1:
            out.append(lead + "  Development Mode:              " + " " * 5 + ("T" if self.dev else "F"))
            lead = ""
        out.append(lead + "  Print Level:                   " + " " * 5 + str(self.prlvl))
        if self.prlvl > 0:
            out += ["", "  __metric__"]
            rec = "  S power:                      " + " " * 5       # (2x,a,5x), advance='no'
            power = {INV: "-1", SQRT_: "0.5", INV_SQRT: "-0.5"}.get(self.metric_type)
            it_line = "  Iterative metric evaluation:  " + " " * 6 + ("T" if self.metric_iterative else "F")
            if power is not None:
                out += [rec + power, it_line]
            else:
                out.append(rec + it_line)
            if self.metric_iterative and self.prlvl > 1:
                out.append("  Number of cycles:             " + " " * 5 + str(self.metric_cycles))
            out += ["", "  __chempot__", "  Initial Chemical Potential:   " + " " * 3 + f"{self.chempot_guess:13.8f}"]
            if self.prlvl > 1:
                out.append("  Number of cycles:             " + " " * 5 + str(self.chempot_cycles))
            out += ["", "  __thresholds_", "  Threshold:                      " + " " * 3 + _fortran_e(thrs_normal, 13, 6)]
        out += ["", "*" * 72, ""]
        return "\n".join(out) + "\n"

    @classmethod
    def from_file(cls, path) -> "PurificationSettings":
        with open(path) as f:
            return cls().read(f.read())


def _pick(table, key, msg):
    if key not in table:
        raise PurSettingsError(msg)
    return table[key]


def _readline(raw: str):
    """Tokens of one settings line as source/readline.f90:1-64 splits them.

    The record is read into an 80-character variable (the rest is dropped),
    split at blanks and tabs, and each token is classed by checktype
    (source/readl2.f90:52-90): a number if it reads as a real, a logical if it
    is exactly ``true`` or ``false`` (dropped here: no setting reads them), a
    string otherwise.  Strings and numbers are numbered separately, so in
    ``cycles = 40`` the value is the first number and ``arg3`` is empty.
    """
    strs, floats = [], []
    for tok in raw[:80].replace("\t", " ").split(" "):
        if not tok:
            continue
        num = _checktype_number(tok)
        if num is not None:
            floats.append(num)
        elif tok not in ("true", "false"):
            strs.append(tok)
    return strs, floats


def _checktype_number(tok: str):
    # a Fortran real field: digits with an optional point and an exponent
    # introduced by e or d (either case).  nan and inf are not taken as numbers:
    # the reference's int() of them is undefined, here they count as strings.
    try:
        v = float(tok.replace("d", "e").replace("D", "e"))
    except ValueError:
        return None
    return v if math.isfinite(v) else None


def _int_value(num: float) -> int:
    """int(floats(1)) of the reference, for a value that fits its 8-byte default integer."""
    if not -2.0 ** 63 <= num < 2.0 ** 63:
        raise PurSettingsError(f"Error: .PUR value {num!r} does not fit an integer setting")
    return int(num)


def _fortran_e(x: float, w: int, d: int) -> str:
    """Fortran Ew.d output: 0.<d digits>E<sign><two digits>, right-justified in w columns."""
    if x == 0.0:
        s = "0." + "0" * d + "E+00"
    else:
        m, e = f"{abs(x):.{d - 1}e}".split("e")
        s = ("-" if x < 0 else "") + "0." + m.replace(".", "") + f"E{int(e) + 1:+03d}"
    return s.rjust(w)
