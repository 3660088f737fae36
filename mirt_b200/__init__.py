"""mirt_b200 -- B200 (sm_100a) implementation of MIRT's table-based NUFFT
interpolation (JeffFessler/mirt nufft/table/) behind the reference's own
interfaces.

* ``mirt_b200.mex``: the eight mex gateways (interp{1,2,3,4}_table[_adj]_mex)
* ``mirt_b200.nufft``: device plans, nufft_init / nufft / nufft_adj, newfft (table mode)
* ``mirt_b200.dcf``: density compensation (ir_mri_density_comp 'pipe', 'jackson')
* ``mirt_b200.learned_dcf``: the learned density compensation (features, MLP)
* ``include/mirt_b200.h``: the C ABI of libmirt_b200.so underneath both

All compute runs in libmirt_b200.so; importing the package does not load it,
calling any compute function does, and fails loudly if it has not been built.
"""
from ._lib import MirtError, load
from .mex import (MexError, interp1_table_adj_mex, interp1_table_mex, interp2_table_adj_mex,
                  interp2_table_mex, interp3_table_adj_mex, interp3_table_mex,
                  interp4_table_adj_mex, interp4_table_mex)
from .nufft import (InterpPlan, NewfftPlan, NufftPlan, minmax_kb_scale, minmax_kb_table, newfft,
                    newfft_kb_scale, newfft_kb_table, newfft_scale, newfft_table, nufft,
                    nufft_adj, nufft_init, nufft_scale, nufft_table)
from .dcf import dcf_jackson, dcf_pipe, ir_mri_density_comp
from .learned_dcf import DcfMLP, LearnedDCF, dcf_features

__all__ = [
    "MirtError", "MexError", "load",
    "interp1_table_mex", "interp2_table_mex", "interp3_table_mex", "interp4_table_mex",
    "interp1_table_adj_mex", "interp2_table_adj_mex", "interp3_table_adj_mex",
    "interp4_table_adj_mex",
    "InterpPlan", "NufftPlan", "minmax_kb_table", "minmax_kb_scale",
    "nufft_init", "nufft", "nufft_adj", "nufft_table", "nufft_scale",
    "NewfftPlan", "newfft", "newfft_kb_table", "newfft_kb_scale", "newfft_table", "newfft_scale",
    "dcf_pipe", "dcf_jackson", "ir_mri_density_comp",
    "dcf_features", "DcfMLP", "LearnedDCF",
]
