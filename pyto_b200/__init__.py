"""pyto_b200: B200-native voxel hex8 structural FEA (drop-in for PyTO's hot path).

Reference-compatible modules: hex_mesher, bound_cond, mat_lib,
topopt_material_model, hex_element_stiffness, hex_structural_fea,
linear_solvers, deflation, topopt_filters, topopt_obj_cons_sensitivities,
topopt_common, topopt_ocm.  Device engine: engine.HexGrid (C ABI of
libpyto_b200.so, sm_100a).
"""
__version__ = "0.1.0"
