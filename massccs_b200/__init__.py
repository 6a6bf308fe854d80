"""massccs_b200: a B200-native engine for the trajectory-method CCS hot path
of cces-cepid/massccs.

    engine.Engine    the C-ABI trajectory engine (include/massccs_gpu.h)
    host.System      the reference's set-up and reduction (include/massccs_host.h)
    synth            seeded synthetic benchmark targets
    build            the in-tree build of the native libraries
"""
__all__ = ["engine", "host", "synth", "build"]
