"""B200-native groundwater (3D Richards) step of frehg2.

The package holds the host side of the drop-in: the reference-shaped
configuration (:mod:`frehg_b200.config`), the ctypes mirror of the C ABI
(:mod:`frehg_b200.abi`) and the :class:`frehg_b200.gw.RichardsSolver`
wrapper.  The step itself runs in ``csrc/`` (CUDA for sm_100a) behind
``include/frehg_gw.h``.
"""
