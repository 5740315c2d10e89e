"""Result and boundary-condition records with the reference's field orders
(src/CutAndDisplaceJulia.jl:46-88).  Greek letters of the Julia names are
spelled in ASCII: εxxDn -> exxDn, σxx -> sxx."""
from __future__ import annotations

from dataclasses import dataclass, fields

import numpy as np


class _Record:
    def __iter__(self):
        return iter(getattr(self, f.name) for f in fields(self))

    def as_list(self):
        return list(self)


@dataclass
class Strains(_Record):
    exx: object = None
    eyy: object = None
    ezz: object = None
    exy: object = None
    exz: object = None
    eyz: object = None


@dataclass
class Disps(_Record):
    Ux: object = None
    Uy: object = None
    Uz: object = None


@dataclass
class Stresses(_Record):
    sxx: object = None
    syy: object = None
    szz: object = None
    sxy: object = None
    sxz: object = None
    syz: object = None


@dataclass
class Tractions(_Record):
    Tn: object = None
    Tss: object = None
    Tds: object = None


@dataclass
class MixedBoundaryConditions(_Record):
    Stresses: Stresses = None
    Tractions: Tractions = None


@dataclass
class FrictionParameters(_Record):
    """Friction coefficient mu (the reference's µ) and cohesion Sf, per
    element or one value for all."""
    mu: object = None
    Sf: object = None


@dataclass
class MixedBoundaryConditionsFriction(_Record):
    MixedBoundaryConditions: MixedBoundaryConditions = None
    FrictionParameters: FrictionParameters = None


@dataclass
class StrainInf(_Record):
    exxDn: object = None
    eyyDn: object = None
    ezzDn: object = None
    exyDn: object = None
    exzDn: object = None
    eyzDn: object = None
    exxDss: object = None
    eyyDss: object = None
    ezzDss: object = None
    exyDss: object = None
    exzDss: object = None
    eyzDss: object = None
    exxDds: object = None
    eyyDds: object = None
    ezzDds: object = None
    exyDds: object = None
    exzDds: object = None
    eyzDds: object = None


@dataclass
class DispInf(_Record):
    DnUx: object = None
    DnUy: object = None
    DnUz: object = None
    DssUx: object = None
    DssUy: object = None
    DssUz: object = None
    DdsUx: object = None
    DdsUy: object = None
    DdsUz: object = None


@dataclass
class TractionInf(_Record):
    DnTn: object = None
    DnTss: object = None
    DnTds: object = None
    DssTn: object = None
    DssTss: object = None
    DssTds: object = None
    DdsTn: object = None
    DdsTss: object = None
    DdsTds: object = None


def empty_like_record(cls):
    return cls(*([np.empty(0)] * len(fields(cls))))


# Elastic constants as typed values (src/CutAndDisplaceJulia.jl:33-37), so that
# ElasticConstantsCheck can tell which two of them it was given.
@dataclass
class PoissonsRatio:
    nu: float


@dataclass
class ShearModulus:
    G: float


@dataclass
class BulkModulus:
    K: float


@dataclass
class YoungsModulus:
    E: float


@dataclass
class LamesConstant:
    lam: float
