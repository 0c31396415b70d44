"""Host-side mirror of hp-multiphysics' tri_hp interface for the B200 library.

The compute path is the C-ABI library lib/libhp_b200.so (CUDA kernels for
sm_100a); this package only prepares meshes, boundary conditions and initial
states and calls the library through ctypes.
"""
from . import _lib
from .mesh import Mesh, square_mesh, delaunay_square, channel_hole, min_angles, read_grd, createsegtri
from .problem import (Problem, GPULevel, basis_tables, kovasznay_ins, lid_cavity_ins, cd_sinsin, cd_quadratic,
                      channel_cylinder_ins, circle_curve, splitmix64_uniform, default_cfl)
