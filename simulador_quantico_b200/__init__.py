"""B200-native state-vector engine for the HybriD-GM t_GPU path.

Hand-written sm_100a CUDA kernels behind the reference's GPU-backend C-ABI
(include/hgm_dropin.h) and a native C-ABI (include/hgm_b200.h).  The
libraries are built in-tree by ``python simulador_quantico_b200/build.py``;
importing this package without them raises ImportError (there is no CPU
fallback).
"""
from .engine import (DGM, T_CPU, T_GPU, T_HYBRID, T_PAR_CPU, Batch, Circuit, PinnedArray, Plan, Server, State, Timer,
                     init, kernel_launches, mem_info, plan_opts, synchronize)
from ._lib import HGM_F32, HGM_F64, HgmError, load_dropin

__all__ = ["DGM", "Batch", "Server", "Circuit", "PinnedArray", "Plan", "State", "Timer", "init", "synchronize",
           "kernel_launches", "mem_info", "plan_opts",
           "load_dropin", "HgmError", "HGM_F32", "HGM_F64", "T_CPU", "T_PAR_CPU", "T_GPU", "T_HYBRID"]
