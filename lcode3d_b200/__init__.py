"""B200-native LCODE 3D quasistatic xi-step solver.

``lcode3d_b200.lcode`` is the drop-in for the reference's ``lcode.py``
module interface (``init``, ``step`` and the stage functions); the device
work runs in ``liblc3d.so`` (C ABI in ``include/lc3d.h``).
"""
from .lcode import (GPUArrays, GPUArraysView, init, step, main,  # noqa: F401
                    move_estimate_wo_fields, move_smart, deposit,
                    initial_deposition, calculate_Ex_Ey_Bx_By, calculate_Ez,
                    calculate_Bz, make_plasma, make_coarse_plasma_grid,
                    make_fine_plasma_grid, solver_for)
