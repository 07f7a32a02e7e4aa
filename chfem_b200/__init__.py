"""chfem_b200 -- B200-native solver hot path of chfem (image-based FEM homogenization).

Public API, with chfem's names:
  compute_property(...)            effective conductivity / stiffness / permeability
  import_nf, import_raw, export_for_chfem   .nf / .raw I/O
  import_{scalar,vector,stress}_field_from_chfem   exported node fields
  compute_conductivity_batch(...)  many images' conductivity tensors in one GPU solve
Native libraries (chfem_b200/lib): libcudapcg_b200.so (GPU solver, drop-in cudapcg C ABI),
libchfem_b200.so (host model layer, femhmg-compatible hmg* API), chfem_exec (CLI).
"""
from .io import (import_nf, import_raw, export_for_chfem, import_scalar_field_from_chfem,
                 import_vector_field_from_chfem, import_stress_field_from_chfem)
from .compute_properties import compute_property
from .batch import compute_conductivity_batch

__all__ = ["compute_property", "compute_conductivity_batch", "import_nf", "import_raw", "export_for_chfem",
           "import_scalar_field_from_chfem", "import_vector_field_from_chfem", "import_stress_field_from_chfem"]
