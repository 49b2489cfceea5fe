"""Sobol generator matrices for the ScrambledSobolSampler path.

The reference sampler (Src/BuiltinComponent/Sampler/ScrambledSobolSampler/Kernel.cpp:20) includes a
generated ``SobolMatrix.dat`` that is not part of its sources (it is git-ignored).  Its comments name
the data set: pbrt's layout (Kernel.cpp:18) built from the Joe & Kuo "new-joe-kuo-6.21201"
direction numbers (ScrambledSobolSampler.cpp:26-27), with ``numSobolDimensions = 1024`` and
``sobolMatrixSize = 52`` (Shared.hpp:22-23).

This module regenerates the three tables that file must provide:

* ``sobolMatrices32[1024 * 52]`` -- column ``c`` of dimension ``d`` is the 32-bit, MSB-aligned
  direction number for index bit ``c``; ``sobolSampleImpl`` XORs the columns selected by the set bits
  of the sample index (Kernel.cpp:23-29).
* ``vdcSobolMatrices[m - 1][c]`` and ``vdcSobolMatricesInv[m - 1][c]`` -- used by
  ``sobolIntervalToIndex`` (Kernel.cpp:31-50) to find the sample index whose first two dimensions fall
  in pixel ``(px, py)`` of a ``2^m x 2^m`` grid.  The first maps frame bit ``c`` (index bit ``2m + c``)
  to its contribution to the pixel code ``(px << m) | py``; the second is the inverse of the
  ``2m x 2m`` map from the low ``2m`` index bits to that code (invertible because dimensions 0/1 form
  a (0,2)-sequence).  Any correct pair of tables yields the same index, so this part is exact.

Direction numbers: the published Joe & Kuo (2008) primitive polynomials and initial values, read
from the copy SciPy ships as data (``scipy/stats/_sobol_direction_numbers.npz``), expanded with the
standard Sobol/Bratley-Fox recurrence
``m_k = 2^s m_{k-s} xor m_{k-s} xor sum_i a_i 2^i m_{k-i}``.  Dimension 0 is van der Corput.

The tables are build artefacts: :func:`write_header` emits a C header that both the CUDA library and
the CPU oracle include, and tests pin its checksum and its (0,2)-net property.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np

NUM_DIMS = 1024
MATRIX_SIZE = 52
VDC_LEVELS = 25  # m = 1 .. 25


def _direction_data():
    import scipy

    path = os.path.join(os.path.dirname(scipy.__file__), "stats", "_sobol_direction_numbers.npz")
    data = np.load(path)
    return data["poly"], data["vinit"]


def sobol_matrices32() -> np.ndarray:
    """Return uint32[NUM_DIMS * MATRIX_SIZE]: column c of dim d at [d * 52 + c]."""
    poly, vinit = _direction_data()
    out = np.zeros((NUM_DIMS, MATRIX_SIZE), dtype=np.uint64)
    for d in range(NUM_DIMS):
        p = int(poly[d])
        s = p.bit_length() - 1  # degree
        m = [0] * (MATRIX_SIZE + 1)  # m[1..52]
        if s == 0:
            for k in range(1, MATRIX_SIZE + 1):
                m[k] = 1
        else:
            for k in range(1, s + 1):
                m[k] = int(vinit[d][k - 1])
            for k in range(s + 1, MATRIX_SIZE + 1):
                v = (m[k - s] << s) ^ m[k - s]
                for i in range(1, s):
                    if (p >> (s - i)) & 1:
                        v ^= m[k - i] << i
                m[k] = v
        for c in range(MATRIX_SIZE):
            k = c + 1
            col = (m[k] << (32 - k)) if k <= 32 else (m[k] >> (k - 32))
            out[d, c] = col & 0xFFFFFFFF
    return out.astype(np.uint32).reshape(-1)


def _pixel_code_column(mat: np.ndarray, c: int, m: int) -> int:
    if c >= MATRIX_SIZE:
        return 0
    x = int(mat[0 * MATRIX_SIZE + c]) >> (32 - m)
    y = int(mat[1 * MATRIX_SIZE + c]) >> (32 - m)
    return (x << m) | y


def _gf2_inverse_columns(cols: list[int], n: int) -> list[int]:
    """Given columns (bit masks of n bits) of an n x n GF(2) matrix A, return columns of A^-1."""
    # Solve A x = e_j for each j by Gaussian elimination on an augmented row representation.
    rows = []
    for r in range(n):
        row = 0
        for c in range(n):
            if (cols[c] >> r) & 1:
                row |= 1 << c
        rows.append([row, 1 << r])  # [A row, identity row]
    piv_row = 0
    where = [-1] * n
    for c in range(n):
        sel = None
        for r in range(piv_row, n):
            if (rows[r][0] >> c) & 1:
                sel = r
                break
        if sel is None:
            raise ValueError("pixel-code matrix is singular")
        rows[piv_row], rows[sel] = rows[sel], rows[piv_row]
        for r in range(n):
            if r != piv_row and (rows[r][0] >> c) & 1:
                rows[r][0] ^= rows[piv_row][0]
                rows[r][1] ^= rows[piv_row][1]
        where[c] = piv_row
        piv_row += 1
    # rows now: row where[c] has A-part == e_c, its identity part = row c of A^-1 (as mask over j)
    inv_rows = [rows[where[c]][1] for c in range(n)]  # inv_rows[c] bit j = Ainv[c][j]
    inv_cols = []
    for j in range(n):
        col = 0
        for c in range(n):
            if (inv_rows[c] >> j) & 1:
                col |= 1 << c
        inv_cols.append(col)
    return inv_cols


def vdc_tables(mat: np.ndarray):
    vdc = np.zeros((VDC_LEVELS, MATRIX_SIZE), dtype=np.uint64)
    vdc_inv = np.zeros((VDC_LEVELS, MATRIX_SIZE), dtype=np.uint64)
    for m in range(1, VDC_LEVELS + 1):
        n = 2 * m
        cols = [_pixel_code_column(mat, c, m) for c in range(n)]
        inv = _gf2_inverse_columns(cols, n)
        for c in range(min(n, MATRIX_SIZE)):
            vdc_inv[m - 1, c] = inv[c]
        for c in range(MATRIX_SIZE):
            vdc[m - 1, c] = _pixel_code_column(mat, n + c, m)
    return vdc, vdc_inv


def tables():
    mat = sobol_matrices32()
    vdc, vdc_inv = vdc_tables(mat)
    return mat, vdc, vdc_inv


def checksum(mat, vdc, vdc_inv) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(mat, dtype="<u4").tobytes())
    h.update(np.ascontiguousarray(vdc, dtype="<u8").tobytes())
    h.update(np.ascontiguousarray(vdc_inv, dtype="<u8").tobytes())
    return h.hexdigest()


def write_header(path: str) -> str:
    """Write the generated tables as a C header; returns the table checksum."""
    mat, vdc, vdc_inv = tables()
    digest = checksum(mat, vdc, vdc_inv)
    lines = [
        "/* Generated by piper2_b200/sobol_tables.py -- do not edit. */",
        "#pragma once",
        "#include <stdint.h>",
        f"#define PB2_SOBOL_DIMS {NUM_DIMS}u",
        f"#define PB2_SOBOL_MATRIX_SIZE {MATRIX_SIZE}u",
        f"#define PB2_SOBOL_VDC_LEVELS {VDC_LEVELS}u",
        f'#define PB2_SOBOL_TABLE_SHA256 "{digest}"',
        "#ifndef PB2_SOBOL_STORAGE",
        "#define PB2_SOBOL_STORAGE static const",
        "#endif",
        f"PB2_SOBOL_STORAGE uint32_t pb2_sobol_matrices32[{NUM_DIMS * MATRIX_SIZE}] = {{",
    ]
    flat = [f"0x{int(v):08x}u" for v in mat]
    for i in range(0, len(flat), 8):
        lines.append("  " + ", ".join(flat[i:i + 8]) + ",")
    lines.append("};")
    for name, arr in (("pb2_vdc_sobol_matrices", vdc), ("pb2_vdc_sobol_matrices_inv", vdc_inv)):
        lines.append(f"PB2_SOBOL_STORAGE uint64_t {name}[{VDC_LEVELS}][{MATRIX_SIZE}] = {{")
        for m in range(VDC_LEVELS):
            vals = [f"0x{int(v):016x}ull" for v in arr[m]]
            lines.append("  {" + ", ".join(vals) + "},")
        lines.append("};")
    text = "\n".join(lines) + "\n"
    old = None
    if os.path.exists(path):
        with open(path) as f:
            old = f.read()
    if old != text:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            f.write(text)
    return digest


if __name__ == "__main__":
    import sys

    print(write_header(sys.argv[1]))
