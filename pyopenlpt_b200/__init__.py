"""B200-native OpenLPT hot path: IPR (peak finding, stereo matching, shake) and the
Shake-the-Box frame loop, as sm_100a CUDA kernels behind a C ABI (include/olpt.h).

``pyopenlpt_b200._ffi`` binds the C ABI with ctypes; ``pyopenlpt_b200.synth``
generates seeded synthetic scenes in the reference's file formats.
"""
__all__ = ["synth"]
