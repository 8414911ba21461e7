"""Loading helpers for the golden fixtures in tests/golden (made by make_golden.py)."""

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["c1_water", "c1_sampled", "mix_small", "silica", "c2_mixture", "c1_retry"]


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


def point_box(lat6, pts):
    """A BoxArrays of single-atom molecules at the given centres on a non-cubic lattice
    (lat6 = alatx, blatx, clatx, blaty, claty, clatz), for the minimum-image goldens; the
    tables are a one-point stub that nothing here evaluates."""
    from epsr_python_translation_b200.box import BoxArrays
    n = pts.shape[0]
    f32 = np.float32
    z1 = np.zeros((1, 4), f32)
    return BoxArrays(
        naf=np.arange(n, dtype=np.int32), nato=np.ones(n, np.int32), mtype=np.zeros(n, np.int32),
        itype=np.zeros(n, np.int32), xa=np.zeros(n, f32), ya=np.zeros(n, f32), za=np.zeros(n, f32),
        xadd=np.ascontiguousarray(pts[:, 0], f32), yadd=np.ascontiguousarray(pts[:, 1], f32),
        zadd=np.ascontiguousarray(pts[:, 2], f32), npairref=np.zeros((1, 1), np.int32),
        n1extr=np.zeros(1, np.int32), n2extr=np.zeros(1, np.int32), nmoltype=1, dmax=f32(1.0),
        cellst=f32(0.03), x=np.zeros(4, f32), xstar=np.zeros(4, f32), npt=3, npt1=2, npt2=1, nptmax=2,
        xavs=z1.copy(), xavs1=z1.copy(), ecoul=z1.copy(), ecoul1=z1.copy(), simt=f32(2.477),
        cfrac=np.ones(1, f32), natomr=n, cubic=False, lat6=np.ascontiguousarray(lat6, f32))
