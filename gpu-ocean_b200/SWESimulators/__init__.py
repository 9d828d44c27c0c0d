"""B200-native CDKLM16 simulator package.

Drop-in for the CDKLM16 path of gpu-ocean's ``SWESimulators`` package
(gpu_ocean/SWESimulators/): the same module names (``Common``,
``Simulator``, ``CDKLM16``, ``WindStress``) and the same public classes,
backed by hand-written sm_100a CUDA reached through a C ABI.
"""
