"""akantu2_b200: the explicit lumped-mass central-difference step of Akantu's
SolidMechanicsModel, as hand-written sm_100a CUDA kernels behind a C ABI
(include/akb_capi.h, libakb.so) with an akantu-style Python binding.
"""
from ._capi import AkbError, LIB_PATH, lib
from .mesh import (Mesh, _hexahedron_8, _tetrahedron_4, _triangle_6, box_hex8, box_tet4,
                   boundary_nodes, gaussian_random_field, square_tri6)
from .server import Server
from .distributed import DistributedModel, PartitionedModel, Subdomain, partition_elements
from .model import (BatchModel, ElementDataMaterialSelector, FixedValue, FromHigherDim,
                    MaterialSelector, MeshDataMaterialSelector, MeshDataMaterialSelectorInt,
                    MeshDataMaterialSelectorString, neumann_forces, Material, SolidMechanicsModel,
                    _explicit_lumped_mass, _x, _y, _z, getStaticParser, parseInput)

__all__ = [
    "AkbError", "BatchModel", "Server", "LIB_PATH", "lib", "Mesh", "_hexahedron_8", "_tetrahedron_4", "_triangle_6",
    "box_hex8", "box_tet4", "boundary_nodes", "gaussian_random_field", "square_tri6", "FixedValue", "FromHigherDim", "neumann_forces", "Material",
    "SolidMechanicsModel", "_explicit_lumped_mass", "_x", "_y", "_z", "getStaticParser",
    "parseInput", "DistributedModel", "PartitionedModel", "Subdomain", "partition_elements",
    "MaterialSelector", "ElementDataMaterialSelector", "MeshDataMaterialSelector",
    "MeshDataMaterialSelectorString", "MeshDataMaterialSelectorInt",
]
