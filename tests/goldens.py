"""Loading helpers for the golden fixtures in tests/golden (made by make_golden.py)."""

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["c1_water", "c1_sampled", "mix_small", "silica", "c2_mixture"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def bits(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.view(np.uint32)


def assert_bits_equal(a, b, what=""):
    """Bitwise float32 equality, with +0 and -0 treated as equal."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    za = (a == 0) & (b == 0)
    diff = (bits(a) != bits(b)) & ~za
    if diff.any():
        idx = np.argwhere(diff)[:5]
        raise AssertionError(f"{what}: {int(diff.sum())} of {a.size} differ, first {idx.tolist()} "
                             f"{a[tuple(idx[0])]!r} vs {b[tuple(idx[0])]!r}")


def golden_cells_csr(z):
    """Reference molsincell(maxcellno, ncell) (1-based) -> CSR (0-based molecules)."""
    n = z["cell_nmolsincell"]
    mols = z["cell_molsincell"]
    start = np.zeros(n.shape[0] + 1, np.int32)
    start[1:] = np.cumsum(n)
    flat = np.zeros(int(start[-1]), np.int32)
    for c in range(n.shape[0]):
        flat[start[c]:start[c + 1]] = mols[: n[c], c] - 1
    return start, flat


def golden_store(z, prefix):
    """Reference store (molergpair[slot, im] 1-based) -> per-molecule partner lists (0-based)
    and energy values in slot order."""
    nm = z[prefix + "nergpairm"]
    mol = z[prefix + "molergpair"]
    ref = z[prefix + "ergpairref"]
    erg = z[prefix + "ergpair"]
    partners, energies = [], []
    for im in range(nm.shape[0]):
        k = nm[im]
        partners.append(mol[:k, im] - 1)
        energies.append(erg[ref[:k, im] - 1])
    return partners, energies
