"""B200-native static-AMR cut-cell explicit time step (HLLC/AUSM+-up, laminar/SA-neg, SRD, SSP-RK3).

The compute path is libamr_b200.so (CUDA, sm_100a) behind the C ABI of include/amr_b200.h;
this package holds the host-side mirrors of that ABI used from Python.
"""
__all__ = ['airfoils', 'cases', 'mesh']
