"""Tolerance comparator of the reference's CI (scripts/compare_output.py:1-93).

TEST INFRASTRUCTURE ONLY.  Restates the reference's acceptance rule for
golden files so the tests accept exactly what the reference's CI accepts:
a value passes if |a-b| <= tol, or if (|a-b|)/b <= tol (note: signed b, as in
scripts/compare_output.py:76); when either value is below tol in magnitude
only the absolute difference counts (:79-82).
"""
from __future__ import annotations


def is_number(s: str) -> bool:
    try:
        float(s)
        return True
    except ValueError:
        return False


def read_data(path: str):
    """Numbers per data line, '=' treated as a separator (scripts/compare_output.py:19-28)."""
    data = []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or line.startswith(" #") or line.startswith("!"):
                continue
            vals = [float(item) for part in line.split("=") for item in part.split() if is_number(item)]
            data.append(vals)
    return data


def compare_rows(rows1, rows2, tol: float = 1.0e-7):
    """Return the list of (line, column, a, b) mismatches under the reference's rule."""
    bad = []
    if len(rows1) != len(rows2):
        return [("lines", len(rows1), len(rows2), None)]
    for ln, (l1, l2) in enumerate(zip(rows1, rows2), start=1):
        if len(l1) != len(l2):
            bad.append(("columns", ln, len(l1), len(l2)))
            continue
        for col, (a, b) in enumerate(zip(l1, l2), start=1):
            if abs(a) > tol and abs(b) > tol:
                if abs(a - b) > tol and abs(a - b) / b > tol:
                    bad.append((ln, col, a, b))
            elif abs(a) < tol or abs(b) < tol:
                if abs(a - b) > tol:
                    bad.append((ln, col, a, b))
    return bad
