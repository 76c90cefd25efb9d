"""tensorkit_b200 — TensorKit.jl's symmetric-contraction path on B200 (sm_100a).

Host mirror of the reference API (1-based leg indices, as in TensorKit) over the libtkb200
C-ABI kernels: sectors and spaces, fusion trees and tree transformers, TensorMap with
device storage, permute/braid/transpose/add_transform!, blockwise mul!/norm/tr/inner,
tensorcontract!/tensoradd! and `tensor("C[..] := A[..]*B[..]")` (@tensor), and the
ChainRules-style rrules with hand-written adjoint kernels.
"""
from .sectors import (U1Irrep, SU2Irrep, ProductSector, Nsymbol, Fsymbol, Rsymbol, Bsymbol,
                      frobenius_schur_phase)
from .spaces import GradedSpace, Vect, ProductSpace, HomSpace, SpaceMismatch, otimes
from .fusiontrees import FusionTree, FusionTreeBlock
from .structure import sectorstructure, degeneracystructure, fusionblocks, subblockstructure
from .treetransformers import treebraider, flatten_transformer, FlatTable
from .tensor import TensorMap, AdjointTensorMap
from .backend import (get_context, set_precision, using_precision, precision, B200Backend,
                      empty_globalcaches, launch_count)
from .indexmanipulations import (permute, permute_, braid, braid_, transpose, transpose_,
                                 repartition, add_transform_, flip)
from .linalg import mul_, compose, norm, tr, inner, dot, scale_, add_
from .tensoroperations import (tensoradd_, tensorcontract_, tensorcontract, contract_,
                               tensor, tensorcontract_structure, tensoradd_structure,
                               tensortrace_, tensortrace, tensortrace_structure)
from .trace import trace_permute_, trace_permute
from .network import NetworkPlan
from . import storage
from .storage import to_dict, from_dict
from . import factorizations
from .factorizations import (svd_compact, svd_vals, svd_trunc, qr_compact, lq_compact, eigh_full,
                             eigh_vals, eigh_trunc, notrunc, truncrank, trunctol, truncerror,
                             truncspace)

__version__ = "0.1.0"
