"""QUICK basis-set arrays, restated from the Fortran reader.

The GPU entry point ``gpu_upload_basis_`` receives some thirty Fortran arrays
that QUICK's ``readbasis`` (src/basis.f90:10-957) and ``xnorm``/``xnewnorm``
(src/subs/xnorm.f90) build from a basis file.  QUICK's Fortran cannot be built
on this image, so this module restates that reader in numpy, shell for shell:
the same shell order (atoms in input order, shells in file order), the same
1-based indices stored inside the arrays (``kstart``, ``katom``, ``Ksumtype``,
``Qsbasis``...), the same Cartesian component order (``KLMN``) and the same
normalisation of the contraction coefficients (``gccoeff``) and components
(``cons``), so that the arrays can be handed unchanged to either this
package's C ABI or the reference's own.

Array shapes follow the Fortran declarations; every 2-D array is stored
column-major (``order='F'``) exactly as the Fortran caller passes it.
"""
import copy
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

MAXPRIM = 10                       # src/modules/quick_size_module.f90:37
PI = 3.1415926535897932384626433832795
PITO3HALF = PI ** 1.5              # src/modules/quick_constants_module.f90:53
# Bohr conversion used when QUICK reads Angstrom input
# (src/modules/quick_constants_module.f90:71-72, applied at
# src/modules/quick_molspec_module_.f90:355).  Note it is 0.529177083, not the
# BOHR parameter 0.5291772083 on line 59 of the same module.
BOHRS_TO_A = 0.529177083
A_TO_BOHRS = 1.0 / BOHRS_TO_A

ATOMIC_NUMBER = {"H": 1, "HE": 2, "LI": 3, "BE": 4, "B": 5, "C": 6, "N": 7,
                 "O": 8, "F": 9, "NE": 10}

# Cartesian components of a d and an f shell in QUICK order with their
# ``cons`` factors (src/basis.f90:546-573 for D, 601-643 for F).
_D_KLMN = [((2, 0, 0), 1.0), ((1, 1, 0), math.sqrt(3.0)), ((0, 2, 0), 1.0),
           ((1, 0, 1), math.sqrt(3.0)), ((0, 1, 1), math.sqrt(3.0)), ((0, 0, 2), 1.0)]
_F_KLMN = [((3, 0, 0), 1.0), ((2, 1, 0), math.sqrt(5.0)), ((1, 2, 0), math.sqrt(5.0)),
           ((0, 3, 0), 1.0), ((2, 0, 1), math.sqrt(5.0)),
           ((1, 1, 1), math.sqrt(5.0) * math.sqrt(3.0)), ((0, 2, 1), math.sqrt(5.0)),
           ((1, 0, 2), math.sqrt(5.0)), ((0, 1, 2), math.sqrt(5.0)), ((0, 0, 3), 1.0)]
# ktype per shell label (number of Cartesian functions), src/basis.f90:390-590
_KTYPE = {"S": 1, "P": 3, "SP": 4, "D": 6, "F": 10}

_DATA = None


def _basis_data():
    global _DATA
    if _DATA is None:
        here = os.path.dirname(os.path.abspath(__file__))
        with open(os.path.join(here, "data", "basis_sets.json")) as fh:
            _DATA = json.load(fh)
    return _DATA


def available_basis_sets():
    return sorted(_basis_data().keys())


def xnorm(a, i, j, k):
    """Primitive normalisation (src/subs/xnorm.f90:26-60)."""
    v = (2.0 * a) ** ((i + j + k) / 2.0 + 0.75)
    gamma = 1.0
    for n in (i, j, k):
        for L in range(1, n + 1):
            gamma = gamma * ((n - L) + 0.5)
    return v * PI ** (-0.75) * gamma ** (-0.5)


def xnewnorm(i, j, k, coeffs, expos):
    """Contracted-function renormalisation (src/subs/xnorm.f90:63-97)."""
    v = 0.0
    xponent = -1.5 + (-i - j - k)
    n = len(coeffs)
    for c1 in range(n):
        for c2 in range(n):
            v = v + coeffs[c1] * coeffs[c2] * (expos[c1] + expos[c2]) ** xponent
    gamma = 1.0
    for m in (i, j, k):
        for L in range(1, m + 1):
            gamma = gamma * ((m - L) + 0.5)
    return (v * gamma * PITO3HALF) ** (-0.5)


@dataclass
class Basis:
    """The arrays ``gpu_upload_basis_`` takes, in QUICK's layout.

    Scalars: natom, nshell, nprim, jshell, jbasis, nbasis, maxcontract.
    Integer arrays keep QUICK's 1-based stored indices.
    """
    natom: int
    nshell: int
    nprim: int
    jshell: int
    jbasis: int
    nbasis: int
    maxcontract: int
    ncontract: np.ndarray       # (nbasis)
    itype: np.ndarray           # (3, nbasis)
    aexp: np.ndarray            # (maxcontract, nbasis)
    dcoeff: np.ndarray          # (maxcontract, nbasis)
    first_basis_function: np.ndarray   # (natom)
    last_basis_function: np.ndarray    # (natom)
    first_shell_basis_function: np.ndarray  # (natom)  (not used on the GPU path)
    last_shell_basis_function: np.ndarray   # (natom)
    ncenter: np.ndarray         # (nbasis)
    kstart: np.ndarray          # (nshell)
    katom: np.ndarray           # (nshell)
    ktype: np.ndarray           # (nshell)
    kprim: np.ndarray           # (nshell)
    kshell: np.ndarray          # (93)
    Ksumtype: np.ndarray        # (nshell+1)
    Qnumber: np.ndarray         # (nshell)
    Qstart: np.ndarray          # (nshell)
    Qfinal: np.ndarray          # (nshell)
    Qsbasis: np.ndarray         # (nshell, 4)  Fortran (nshell, 0:3)
    Qfbasis: np.ndarray         # (nshell, 4)
    gccoeff: np.ndarray         # (MAXPRIM, nbasis)
    cons: np.ndarray            # (nbasis)
    gcexpo: np.ndarray          # (MAXPRIM, nbasis)
    KLMN: np.ndarray            # (3, nbasis)
    gcexpomin: np.ndarray = field(default=None)  # (nshell)

    @property
    def max_l(self):
        return int(self.Qfinal.max())


_BASIS_CACHE = {}


def build_basis(atoms, basis_name):
    """Build QUICK's basis arrays for ``atoms`` (list of element symbols).

    Follows readbasis' second pass (src/basis.f90:376-757) shell by shell and
    its post-processing (src/basis.f90:797-897).  The arrays depend only on
    the element list and the basis name: each distinct (elements, basis) is
    built once per process and later calls get their own copy.
    """
    key = (tuple(a.upper() for a in atoms), basis_name)
    if key not in _BASIS_CACHE:
        if len(_BASIS_CACHE) > 256:
            _BASIS_CACHE.clear()
        _BASIS_CACHE[key] = _build_basis(atoms, basis_name)
    return copy.deepcopy(_BASIS_CACHE[key])


def _build_basis(atoms, basis_name):
    """build_basis without the cache."""
    data = _basis_data()[basis_name]
    atoms = [a.upper() for a in atoms]
    natom = len(atoms)
    # first pass: sizes (src/basis.f90:54-96, 166-200)
    nshell = nbasis = nprim = 0
    for a in atoms:
        for sh in data[a]:
            nshell += 1
            nbasis += _KTYPE[sh["label"]]
            nprim += len(sh["prims"])

    f64 = lambda *s: np.zeros(s, dtype=np.float64, order="F")
    i32 = lambda *s: np.zeros(s, dtype=np.int32, order="F")
    kstart, katom, ktype, kprim = i32(nshell), i32(nshell), i32(nshell), i32(nshell)
    Ksumtype = i32(nshell + 1)
    Qnumber, Qstart, Qfinal = i32(nshell), i32(nshell), i32(nshell)
    Qsbasis, Qfbasis = i32(nshell, 4), i32(nshell, 4)
    gccoeff, gcexpo = f64(MAXPRIM, nbasis), f64(MAXPRIM, nbasis)
    cons, KLMN = f64(nbasis), i32(3, nbasis)
    gcexpomin = np.full(nshell, 99999.0)
    aex = np.zeros(nprim)
    gcs, gcp, gcd, gcf = (np.zeros(nprim) for _ in range(4))
    kshell = i32(93)
    for a in set(atoms):
        kshell[ATOMIC_NUMBER[a] - 1] = len(data[a])

    jbasis = 1       # next primitive (1-based)
    jshell = 1       # next shell (1-based)
    ninit = 0        # last basis function assigned (1-based count)
    for iat, a in enumerate(atoms, start=1):
        for sh in data[a]:
            label = sh["label"]
            prims = sh["prims"]
            iprim = len(prims)
            s = jshell - 1
            kprim[s] = iprim
            katom[s] = iat
            kstart[s] = jbasis
            ktype[s] = _KTYPE[label]
            Ksumtype[s] = ninit + 1
            AA = [float(p[0]) for p in prims]
            BB = [float(p[1]) for p in prims]
            CC = [float(p[2]) for p in prims] if label == "SP" else None
            for k in range(iprim):
                aex[jbasis - 1 + k] = AA[k]
                if label == "S":
                    gcs[jbasis - 1 + k] = BB[k]
                elif label == "P":
                    gcp[jbasis - 1 + k] = BB[k]
                elif label == "SP":
                    gcs[jbasis - 1 + k] = BB[k]
                    gcp[jbasis - 1 + k] = CC[k]
                elif label == "D":
                    gcd[jbasis - 1 + k] = BB[k]
                elif label == "F":
                    gcf[jbasis - 1 + k] = BB[k]
            jbasis += iprim
            gcexpomin[s] = min(gcexpomin[s], min(AA))

            def fill(col, klmn, coef):
                for k in range(iprim):
                    gccoeff[k, col] = coef[k] * xnorm(AA[k], *klmn)
                    gcexpo[k, col] = AA[k]

            if label == "S":                       # src/basis.f90:406-435
                Qnumber[s], Qstart[s], Qfinal[s] = 0, 0, 0
                Qsbasis[s, 0], Qfbasis[s, 0] = 0, 0
                ninit += 1
                cons[ninit - 1] = 1.0
                fill(ninit - 1, (0, 0, 0), BB)
                nn = xnewnorm(0, 0, 0, gccoeff[:iprim, ninit - 1], gcexpo[:iprim, ninit - 1])
                gccoeff[:iprim, ninit - 1] *= nn
            elif label == "P":                     # src/basis.f90:436-475
                Qnumber[s], Qstart[s], Qfinal[s] = 6, 1, 1
                Qsbasis[s, 1], Qfbasis[s, 1] = 0, 2
                for c in range(3):
                    ninit += 1
                    cons[ninit - 1] = 1.0
                    KLMN[c, ninit - 1] = 1
                    fill(ninit - 1, (1, 0, 0), BB)
                nn = xnewnorm(1, 0, 0, gccoeff[:iprim, ninit - 1], gcexpo[:iprim, ninit - 1])
                gccoeff[:iprim, ninit - 3:ninit] *= nn
            elif label == "SP":                    # src/basis.f90:476-537
                Qnumber[s], Qstart[s], Qfinal[s] = 1, 0, 1
                Qsbasis[s, 0], Qfbasis[s, 0] = 0, 0
                Qsbasis[s, 1], Qfbasis[s, 1] = 1, 3
                ninit += 1
                cons[ninit - 1] = 1.0
                fill(ninit - 1, (0, 0, 0), BB)
                nn = xnewnorm(0, 0, 0, gccoeff[:iprim, ninit - 1], gcexpo[:iprim, ninit - 1])
                gccoeff[:iprim, ninit - 1] *= nn
                for c in range(3):
                    ninit += 1
                    cons[ninit - 1] = 1.0
                    KLMN[c, ninit - 1] = 1
                    fill(ninit - 1, (1, 0, 0), CC)
                nn = xnewnorm(1, 0, 0, gccoeff[:iprim, ninit - 1], gcexpo[:iprim, ninit - 1])
                gccoeff[:iprim, ninit - 3:ninit] *= nn
            elif label == "D":                     # src/basis.f90:538-598
                Qnumber[s], Qstart[s], Qfinal[s] = 2, 2, 2
                Qsbasis[s, 2], Qfbasis[s, 2] = 0, 5
                for klmn, cf in _D_KLMN:
                    ninit += 1
                    KLMN[:, ninit - 1] = klmn
                    cons[ninit - 1] = cf
                    fill(ninit - 1, klmn, BB)
                # the (2,0,0) norm from the 3rd component scales components
                # 1-3, the (1,1,0) norm from the 6th scales 4-6
                # (src/basis.f90:587-598)
                nn = xnewnorm(2, 0, 0, gccoeff[:iprim, ninit - 4], gcexpo[:iprim, ninit - 4])
                gccoeff[:iprim, ninit - 6:ninit - 3] *= nn
                nn = xnewnorm(1, 1, 0, gccoeff[:iprim, ninit - 1], gcexpo[:iprim, ninit - 1])
                gccoeff[:iprim, ninit - 3:ninit] *= nn
            elif label == "F":                     # src/basis.f90:599-655 (no renormalisation)
                Qnumber[s], Qstart[s], Qfinal[s] = 3, 3, 3
                Qsbasis[s, 3], Qfbasis[s, 3] = 0, 9
                for klmn, cf in _F_KLMN:
                    ninit += 1
                    KLMN[:, ninit - 1] = klmn
                    cons[ninit - 1] = cf
                    fill(ninit - 1, klmn, BB)
            else:
                raise ValueError("unsupported shell label %r" % label)
            jshell += 1
    Ksumtype[jshell - 1] = ninit + 1          # src/basis.f90:746
    jshell -= 1
    jbasis -= 1
    assert jshell == nshell and jbasis == nprim and ninit == nbasis
    maxcontract = int(kprim.max())

    # post-processing (src/basis.f90:797-897)
    ncontract, ncenter = i32(nbasis), i32(nbasis)
    itype = i32(3, nbasis)
    aexp, dcoeff = f64(maxcontract, nbasis), f64(maxcontract, nbasis)
    l = 0
    for i in range(nshell):
        kt = ktype[i]
        for j in range(1, kt + 1):
            ncenter[l] = katom[i]
            ncontract[l] = kprim[i]
            if kt == 3:
                itype[j - 1, l] = 1
            elif kt == 4 and j > 1:
                itype[j - 2, l] = 1
            elif kt == 6:
                itype[:, l] = _D_KLMN[j - 1][0]
            elif kt == 10:
                itype[:, l] = _F_KLMN[j - 1][0]
            for ll, k in enumerate(range(kstart[i] - 1, kstart[i] - 1 + kprim[i])):
                aexp[ll, l] = aex[k]
                if kt == 1:
                    dcoeff[ll, l] = gcs[k]
                elif kt == 3:
                    dcoeff[ll, l] = gcp[k]
                elif kt == 4:
                    dcoeff[ll, l] = gcs[k] if j == 1 else gcp[k]
                elif kt == 6:
                    dcoeff[ll, l] = gcd[k]
                else:
                    dcoeff[ll, l] = gcf[k]
            l += 1
    first_bf, last_bf = i32(natom), i32(natom)
    iatm, is_ = 1, 0
    first_bf[0] = 1
    for i in range(nshell):
        is_ += ktype[i]
        if katom[i] != iatm:
            iatm = katom[i]
            first_bf[iatm - 1] = is_
            last_bf[iatm - 2] = is_ - 1
    last_bf[iatm - 1] = nbasis

    # getMol (src/getMol.f90:85) folds the normalisation into dcoeff before
    # main.f90:168 uploads it; the XC quadrature evaluates basis functions
    # from these coefficients.
    normalize_dcoeff(ncontract, itype, aexp, dcoeff)

    return Basis(natom=natom, nshell=nshell, nprim=nprim, jshell=jshell, jbasis=jbasis,
                 nbasis=nbasis, maxcontract=maxcontract, ncontract=ncontract, itype=itype,
                 aexp=aexp, dcoeff=dcoeff, first_basis_function=first_bf,
                 last_basis_function=last_bf, first_shell_basis_function=i32(natom),
                 last_shell_basis_function=i32(natom), ncenter=ncenter, kstart=kstart,
                 katom=katom, ktype=ktype, kprim=kprim, kshell=kshell, Ksumtype=Ksumtype,
                 Qnumber=Qnumber, Qstart=Qstart, Qfinal=Qfinal, Qsbasis=Qsbasis,
                 Qfbasis=Qfbasis, gccoeff=gccoeff, cons=cons, gcexpo=gcexpo, KLMN=KLMN,
                 gcexpomin=gcexpomin)


def normalize_dcoeff(ncontract, itype, aexp, dcoeff):
    """In-place restatement of normalize_basis
    (src/modules/quick_basis_module_.f90:331-373): primitive norms, then the
    contracted renormalisation, applied to dcoeff column by column."""
    nbasis = dcoeff.shape[1]
    for jb in range(nbasis):
        i, j, k = (int(v) for v in itype[:, jb])
        for c in range(int(ncontract[jb])):
            dcoeff[c, jb] = dcoeff[c, jb] * xnorm(aexp[c, jb], i, j, k)
    for ib in range(nbasis):
        i, j, k = (int(v) for v in itype[:, ib])
        n = int(ncontract[ib])
        xponent = -1.5 + float(-i - j - k)
        v = 0.0
        for c1 in range(n):
            for c2 in range(n):
                v = v + dcoeff[c1, ib] * dcoeff[c2, ib] * (aexp[c1, ib] + aexp[c2, ib]) ** xponent
        gamma = 1.0
        for m in (i, j, k):
            for L in range(1, m + 1):
                gamma = gamma * ((m - L) + 0.5)
        v = (v * gamma * PITO3HALF) ** (-0.5)
        for c in range(n):
            dcoeff[c, ib] = v * dcoeff[c, ib]


def sigrad2(basis, basis_cutoff=1.0e-10):
    """Squared radius of significance per basis function, restating get_sigrad
    (src/dft.f90:536-612): the radius where r^L exp(-a_min r^2) first falls
    below basis_cutoff / sqrt((2 a_min)^(L+3/2) / (2 pi Gamma(L+3/2))),
    located by the same decimal step search (1, 0.1, ... 1e-4)."""
    out = np.zeros(basis.nbasis)
    for ib in range(basis.nbasis):
        amin = 10.0e10
        for c in range(int(basis.ncontract[ib])):
            amin = min(amin, basis.aexp[c, ib])
        L = int(basis.itype[:, ib].sum())
        gamma = 1.0
        for i in range(1, L + 2):
            gamma = gamma * ((L + 1 - i) + 0.5)
        gamma2pi = gamma * 11.13665599366341569
        target = basis_cutoff * (((2.0 * amin) ** (L + 1.5)) / gamma2pi) ** (-0.5)
        step, radial = 1.0, 0.0
        while step > 1.0e-4:
            radial = radial + step
            current = math.exp(-amin * radial * radial) * radial ** L
            if current < target:
                radial = radial - step
                step = step / 10.0
        out[ib] = radial * radial
    return out
