"""B200-native (sm_100a) forward/back projector pair of TRTT.

The CUDA kernels and the drop-in C ABI live in ``libtrtt_b200.so`` (built
from ``csrc/`` by ``build.py``); the modules here are the host side:
``dropin`` (the reference plugin symbols on numpy arrays), ``projectors``
(batched plans, 4D gates, CUDA graphs), ``geometry`` / ``footprint`` (scan
and footprint-table builders), ``recon`` (VMLM-B + TV), ``unet`` /
``warmstart`` (learned warm start), ``phantoms`` / ``workloads`` (seeded
synthetic inputs), ``analytic`` / ``rawio`` (analytic projections and data
files), ``dist`` (view sharding over ranks).
"""
