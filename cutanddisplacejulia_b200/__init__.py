"""B200-native triangular-dislocation (TD) path of CutAndDisplaceJulia.

The hot path -- TD strain / displacement influence of every triangle on every
observation point (full and half space), the traction influence assembly and
the dense slip solve -- runs in libcad_td.so (CUDA, sm_100a) behind a C ABI
(include/cad_td.h).  This package is the Python host mirror of the
reference's Julia interface (same function names, argument order, field
orders and error messages); julia/CutAndDisplaceB200.jl is the Julia one.
"""
from ._lib import CadError, context, load  # noqa: F401
from .assembly import (CalculateInfluenceMatrices3D, CalculateNormalAndShearTractions3D,  # noqa: F401
                       FrictionSolver, KnockOutFixedRows, RemoveFixedElements3D, SetupTractionVector, SlipCalculator3D,
                       SlipCalculator3D_batched, fischer_newton, solve)
from .geometry import (AreaOfTriangle3D, CalculateNormalTraction3D, CalculateSSandDSDirs,  # noqa: F401
                       CalculateTractionInChosenDirection3D, CreateFaceNormalAndMidPoint, CreateP1P2P3,
                       ElasticConstantsCheck, HookesLaw3DStrain2Stress, TensorTransformation3D,
                       TractionVectorCartesianComponents3D)
from .structs import (BulkModulus, DispInf, Disps, FrictionParameters, LamesConstant,  # noqa: F401
                      MixedBoundaryConditions, MixedBoundaryConditionsFriction, PoissonsRatio, ShearModulus,
                      StrainInf, Strains, Stresses, TractionInf, Tractions, YoungsModulus)
from .td import TD, TD_sum  # noqa: F401

__version__ = "1.0.0"
