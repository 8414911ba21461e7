"""Host-side description of one EPSR box: the arrays the pair path reads and writes.

``BoxArrays`` is plain NumPy (0-based molecules/atoms/types/pairs; the r-grid index keeps
the reference's 1-based meaning).  It is built from a synthetic ``configs.System``, from a
golden fixture, or from the reference's COMMON blocks (see ``dropin``), and it is what the
device state (``device.DeviceBox``) is uploaded from and downloaded into.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

f32 = np.float32


@dataclass
class BoxArrays:
    naf: np.ndarray
    nato: np.ndarray
    mtype: np.ndarray
    itype: np.ndarray
    xa: np.ndarray
    ya: np.ndarray
    za: np.ndarray
    xadd: np.ndarray
    yadd: np.ndarray
    zadd: np.ndarray
    npairref: np.ndarray          # (ntype, ntype) 0-based pair index
    n1extr: np.ndarray
    n2extr: np.ndarray
    nmoltype: int
    dmax: np.float32
    cellst: np.float32
    x: np.ndarray                 # r grid (npt+1), 1-based
    xstar: np.ndarray             # (npt+1)
    npt: int
    npt1: int
    npt2: int
    nptmax: int
    xavs: np.ndarray
    xavs1: np.ndarray
    ecoul: np.ndarray
    ecoul1: np.ndarray            # (npairs, npt+1)
    simt: np.float32
    cfrac: np.ndarray             # (ntype,)
    natomr: int
    cubic: bool = True
    lat6: np.ndarray = field(default_factory=lambda: np.array([1, 0, 0, 1, 0, 1], dtype=f32))
    lat9: np.ndarray = field(default_factory=lambda: np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], dtype=f32))
    maxmolsize: np.float32 = f32(0.0)

    @property
    def nmol(self) -> int:
        return int(self.naf.shape[0])

    @property
    def natom(self) -> int:
        return int(self.itype.shape[0])

    @property
    def ntype(self) -> int:
        return int(self.npairref.shape[0])

    @property
    def npairs(self) -> int:
        return int(self.n1extr.shape[0])

    @property
    def stepcl(self) -> np.float32:
        """cellst/dmax in float32 (molfit.py:836, ato_manipulation_rev4.py:3694)."""
        return f32(self.cellst) / f32(self.dmax)

    @property
    def sepmax(self) -> np.float32:
        """Cell-list range of the epsr loop (epsr_standalone_rev3.py:1259)."""
        return self.xstar[self.nptmax] + self.maxmolsize + f32(3.0) / f32(self.dmax)

    def copy(self) -> "BoxArrays":
        kw = {}
        for k, v in self.__dict__.items():
            kw[k] = v.copy() if isinstance(v, np.ndarray) else v
        return BoxArrays(**kw)

    # ------------------------------------------------------------------ constructors
    @staticmethod
    def from_system(s) -> "BoxArrays":
        g = s.grid
        return BoxArrays(
            naf=s.naf.astype(np.int32), nato=s.nato.astype(np.int32), mtype=s.mtype.astype(np.int32),
            itype=s.itype.astype(np.int32), xa=s.xa.astype(f32).copy(), ya=s.ya.astype(f32).copy(),
            za=s.za.astype(f32).copy(), xadd=s.xadd.astype(f32).copy(), yadd=s.yadd.astype(f32).copy(),
            zadd=s.zadd.astype(f32).copy(), npairref=s.npairref.astype(np.int32),
            n1extr=s.n1extr.astype(np.int32), n2extr=s.n2extr.astype(np.int32), nmoltype=int(s.nmoltype),
            dmax=f32(s.dmax), cellst=f32(s.cellst), x=g["x"].astype(f32), xstar=s.xstar.astype(f32),
            npt=int(g["npt"]), npt1=int(g["npt1"]), npt2=int(g["npt2"]), nptmax=int(g["nptmax"]),
            xavs=s.xavs.astype(f32), xavs1=s.xavs1.astype(f32), ecoul=s.ecoul.astype(f32),
            ecoul1=s.ecoul1.astype(f32), simt=f32(s.simt), cfrac=s.cfrac.astype(f32), natomr=int(s.natom),
            maxmolsize=f32(max(float(np.max(np.abs(np.stack([s.xa, s.ya, s.za])))), 0.0) * 2.0))

    @staticmethod
    def from_golden(z) -> "BoxArrays":
        """From a tests/golden/*.npz produced by make_golden.py (the ``sys_*`` inputs)."""
        return BoxArrays(
            naf=z["sys_naf"].astype(np.int32), nato=z["sys_nato"].astype(np.int32),
            mtype=z["sys_mtype"].astype(np.int32), itype=z["sys_itype"].astype(np.int32),
            xa=z["sys_xa"].copy(), ya=z["sys_ya"].copy(), za=z["sys_za"].copy(), xadd=z["sys_xadd"].copy(),
            yadd=z["sys_yadd"].copy(), zadd=z["sys_zadd"].copy(), npairref=z["sys_npairref"].astype(np.int32),
            n1extr=z["sys_n1extr"].astype(np.int32), n2extr=z["sys_n2extr"].astype(np.int32),
            nmoltype=int(z["sys_nmoltype"]), dmax=f32(z["sys_dmax"]), cellst=f32(z["sys_cellst"]),
            x=z["sys_x"].copy(), xstar=z["sys_xstar"].copy(), npt=int(z["sys_npt"]), npt1=int(z["sys_npt1"]),
            npt2=int(z["sys_npt2"]), nptmax=int(z["sys_nptmax"]), xavs=z["sys_xavs"].copy(),
            xavs1=z["sys_xavs1"].copy(), ecoul=z["sys_ecoul"].copy(), ecoul1=z["sys_ecoul1"].copy(),
            simt=f32(z["sys_simt"]), cfrac=z["sys_cfrac"].copy(), natomr=int(z["in_natomr"]),
            maxmolsize=f32(z["in_maxmolsize"]))


@dataclass
class Ran1State:
    """The ran1 COMMON block /ran1com/ (common/ran1com.py): mcall, idum, iy, iv(32)."""
    idum: int = 0
    iy: int = 0
    mcall: int = 0
    iv: np.ndarray = field(default_factory=lambda: np.zeros(32, dtype=np.int32))

    def as_array(self) -> np.ndarray:
        """Packed int32[35]: idum, iy, mcall, iv[0..31] (the device layout)."""
        out = np.zeros(35, dtype=np.int32)
        out[0] = np.int32(self.idum)
        out[1] = np.int32(self.iy)
        out[2] = np.int32(np.int64(self.mcall).astype(np.int32))
        out[3:] = self.iv
        return out

    @staticmethod
    def from_array(a) -> "Ran1State":
        a = np.asarray(a, dtype=np.int32)
        return Ran1State(int(a[0]), int(a[1]), int(a[2]), a[3:35].copy())

    @staticmethod
    def from_golden(z, prefix) -> "Ran1State":
        return Ran1State(int(z[prefix + "idum"]), int(z[prefix + "iy"]), int(z[prefix + "mcall"]),
                         z[prefix + "iv"].astype(np.int32).copy())


_libm = None


def _powf(x, y):
    """glibc powf, the function the reference calls through ctypes (fortran/fmath.py:137)."""
    global _libm
    if _libm is None:
        import ctypes
        import ctypes.util
        _libm = ctypes.CDLL(ctypes.util.find_library("m"))
        _libm.powf.restype = ctypes.c_float
        _libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
    return f32(_libm.powf(float(x), float(y)))


def libm_f1(name, x):
    """glibc's float function ``name`` (cosf, sinf, ...) of x, the function the reference calls
    through ctypes (fortran/fmath.py:67)."""
    import ctypes
    _powf(f32(1.0), f32(1.0))   # loads the library
    fn = getattr(_libm, name)
    fn.restype = ctypes.c_float
    fn.argtypes = [ctypes.c_float]
    return f32(fn(float(x)))


def trsteps(natomr: int):
    """Largest and smallest translational step of molfit (molfit.py:96-101), float32."""
    tmax = _powf(f32(1.0) / f32(natomr), f32(1.0) / f32(3.0))
    tmin = max(f32(0.0001) * tmax, f32(1.0e-6))
    return f32(tmax), f32(tmin)
