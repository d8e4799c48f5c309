"""Residue alphabets of the TOPAZ search path.

Three encodings meet on the path:

* amino-acid letters as they appear in FASTA ("ACDEF...");
* the internal alphabet of the DB text and of queries: 'A'..'Y' stand for
  the amino acids ``INTERNAL_TO_AA`` in that order, and '\\n' delimits
  proteins (``aa2internal``/``internal2aa`` in src/lexicographical.h:95-192);
* substitution-matrix indices 0..24 in ``MATRIX_ORDER`` (the row order of the
  tables in src/substitution.h; ``aa_table2`` in src/lexicographical.h:19-33
  maps internal letters to them).
"""
import numpy as np

INTERNAL_TO_AA = "ACMLJIVTSKRQZEDBNHYFWXP*G"
MATRIX_ORDER = "ARNDCQEGHILKMFPSTWYVBJZX*"
AMINO20 = "ARNDCQEGHILKMFPSTWYV"

# upper_aa (src/lexicographical.h:35-58): A..Y, '*' and '\n' pass, lower case
# a..y is upper-cased, anything else becomes 'X'.
_UPPER = np.full(256, ord("X"), dtype=np.uint8)
for _c in range(ord("A"), ord("Y") + 1):
    _UPPER[_c] = _c
for _c in range(ord("a"), ord("y") + 1):
    _UPPER[_c] = _c - 32
_UPPER[ord("*")] = ord("*")
_UPPER[ord("\n")] = ord("\n")

# aa2internal for upper-case input (src/lexicographical.h:135-161); anything
# without an entry maps to 'V' (internal X).
_AA2INT = np.full(256, ord("V"), dtype=np.uint8)
for _i, _aa in enumerate(INTERNAL_TO_AA):
    _AA2INT[ord(_aa)] = ord("A") + _i
_AA2INT[ord("\n")] = ord("\n")

# internal letter -> matrix index (aa_table2); every other byte -> 23 (X)
_INT2IDX = np.full(256, 23, dtype=np.int8)
for _i, _aa in enumerate(INTERNAL_TO_AA):
    _INT2IDX[ord("A") + _i] = MATRIX_ORDER.index(_aa)
    _INT2IDX[ord("a") + _i] = MATRIX_ORDER.index(_aa)

# amino-acid letter -> matrix index
_AA2IDX = _INT2IDX[_AA2INT]


def upper_aa(b: np.ndarray) -> np.ndarray:
    return _UPPER[np.asarray(b, dtype=np.uint8)]


def aa_to_internal(b: np.ndarray) -> np.ndarray:
    """Upper-cased amino-acid bytes -> internal alphabet bytes."""
    return _AA2INT[np.asarray(b, dtype=np.uint8)]


def internal_to_index(b: np.ndarray) -> np.ndarray:
    """Internal alphabet bytes -> substitution-matrix indices (int8)."""
    return _INT2IDX[np.asarray(b, dtype=np.uint8)]


def aa_to_index(b: np.ndarray) -> np.ndarray:
    """Upper-cased amino-acid bytes -> substitution-matrix indices (int8)."""
    return _AA2IDX[np.asarray(b, dtype=np.uint8)]
