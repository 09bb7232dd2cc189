"""ctypes binding of the engine's C ABI (include/dolfin_b200.h).

The shared library is built in-tree (``dolfin_b200/_lib/libdolfin_b200.so``,
see ``dolfin_b200/build.py``).  There is no fallback: if the library is
missing, importing the engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DOLFIN_B200_LIB") or os.path.join(_HERE, "_lib", "libdolfin_b200.so")

DB2_OK = 0
ERR_NAMES = {1: "argument", 2: "shape", 3: "index", 4: "mesh", 5: "unsupported", 6: "cuda",
             7: "out of memory", 8: "timeout"}

FORM_DIFFUSION, FORM_LOAD, FORM_ELASTICITY = 1, 2, 3
FORM_FACET_MASS, FORM_FACET_LOAD, FORM_FUNCTIONAL, FORM_FACET_FUNCTIONAL = 4, 5, 6, 7
COEFF_NONE, COEFF_CONSTANT, COEFF_P1, COEFF_P1_SCALED, COEFF_COORD, COEFF_P1_KAPPA = 0, 1, 2, 3, 4, 5
FP64, FP32_CONTRACT, FP32_TENSOR_CORE = 0, 1, 2


class DB2Form(C.Structure):
    _fields_ = [("kind", C.c_int), ("coeff", C.c_int), ("constant", C.c_double * 3),
                ("mu", C.c_double), ("lmbda", C.c_double)]


class DB2Error(RuntimeError):
    """Raised for a non-zero status of a C entry point (dolfin_error analogue)."""

    def __init__(self, code, func, msg):
        super().__init__(f"*** Error in {func}: {msg} [{ERR_NAMES.get(code, code)}]")
        self.code = code


_lib = None
P, I, I64, D = C.c_void_p, C.c_int, C.c_int64, C.c_double
PP = C.POINTER(C.c_void_p)

# name -> argtypes (all return int status unless listed in _RESTYPES)
_SIGS = {
    "db2_last_error": [],
    "db2_version": [],
    "db2_kernel_launches": [],
    "db2_mesh_create": [I, I64, P, I64, P, PP],
    "db2_mesh_unit_cube": [I, I, I, PP],
    "db2_mesh_unit_square": [I, I, I, PP],
    "db2_mesh_info": [P, C.POINTER(I), C.POINTER(I64), C.POINTER(I64)],
    "db2_mesh_copy": [P, P, P],
    "db2_mesh_set_coordinates": [P, P],
    "db2_mesh_num_edges": [P, C.POINTER(I64)],
    "db2_mesh_num_exterior_facets": [P, C.POINTER(I64)],
    "db2_mesh_exterior_facets": [P, P, P],
    "db2_mesh_destroy": [P],
    "db2_mesh_read_xml": [C.c_char_p, PP],
    "db2_mesh_write_xml": [P, C.c_char_p],
    "db2_mesh_read_xdmf": [C.c_char_p, PP],
    "db2_pattern_set_row_range": [P, C.c_int64, C.c_int64],
    "db2_pattern_set_row_block": [P, C.c_int64, C.c_int64],
    "db2_tensor_core_status": [P],
    "db2_pattern_row_block_info": [P, P, P],
    "db2_pattern_row_block_csr_host": [P, P, P],
    "db2_mesh_write_xdmf": [P, C.c_char_p, P, C.c_int, C.c_char_p],
    "db2_vector_write_xml": [C.c_char_p, I64, P],
    "db2_vector_read_xml": [C.c_char_p, C.POINTER(I64), P],
    "db2_space_create": [P, I, I, PP],
    "db2_space_create_reordered": [P, I, I, PP],
    "db2_space_node_numbers": [P, P],
    "db2_space_info": [P, C.POINTER(I), C.POINTER(I64)],
    "db2_space_cell_dofs": [P, P],
    "db2_space_destroy": [P],
    "db2_pattern_create": [P, I, PP],
    "db2_pattern_info": [P, C.POINTER(I64), C.POINTER(I64)],
    "db2_pattern_csr_device": [P, PP, PP],
    "db2_pattern_csr_host": [P, P, P],
    "db2_pattern_plan_info": [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I), C.POINTER(I64),
                              C.POINTER(I64), C.POINTER(I64)],
    "db2_pattern_plan_copy": [P, P, P, P, P, P, P],
    "db2_pattern_retile": [P, I, I],
    "db2_pattern_facet_plan_info": [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I)],
    "db2_pattern_facet_plan_copy": [P, P, P, P, P],
    "db2_pattern_destroy": [P],
    "db2_assemble_matrix": [P, P, P, I, P, I, P],
    "db2_assemble_vector": [P, P, P, P, I, P],
    "db2_assemble_system": [P, P, P, P, P, I, P, P, P],
    "db2_assemble_system_bc": [P, P, P, P, P, P, P, I, P, P, P],
    "db2_assemble_scalar": [P, P, P, P, P],
    "db2_assemble_local": [P, P, P, P, P, I64, P, P, P],
    "db2_assemble_facets_bc": [P, P, P, P, P, P, P, P, P, P],
    "db2_apply": [P, P, P, I, P, P, P],
    "db2_vjp_kappa": [P, P, P, P, P, P, P, I, P, P],
    "db2_vjp_kappa_noalloc": [P, P, P, P, P, P, P, I, P, P],
    "db2_batch_create": [I, P, P, P, P, I, I, I, PP],
    "db2_batch_info": [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I)],
    "db2_batch_assemble": [P, I, P],
    "db2_batch_assemble_loop": [P, I, P],
    "db2_batch_destroy": [P],
}
_RESTYPES = {"db2_last_error": C.c_char_p, "db2_version": C.c_char_p,
             "db2_kernel_launches": C.c_int64}


def lib():
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"dolfin_b200 engine library not built ({LIB_PATH}); run "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`make -C dolfin_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def call(name, *args):
    """Call a status-returning entry point; raise DB2Error on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != DB2_OK:
        msg = lib().db2_last_error().decode(errors="replace")
        raise DB2Error(rc, name, msg)
    return rc


def exported_symbols():
    return sorted(_SIGS)


def kernel_launches():
    return int(lib().db2_kernel_launches())


def make_form(kind, coeff=COEFF_NONE, constant=(0.0, 0.0, 0.0), mu=0.0, lmbda=0.0):
    f = DB2Form()
    f.kind, f.coeff = int(kind), int(coeff)
    for i in range(3):
        f.constant[i] = float(constant[i]) if i < len(constant) else 0.0
    f.mu, f.lmbda = float(mu), float(lmbda)
    return f
