"""axon_b200: B200-native engine for AXON's sparse binary assembly network.

The product is ``_build/libaxon_b200.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/axon_capi.h``) and the ``_build/axon`` command line that replaces the
reference's ``build/axon``. This package is the Python side of the same C ABI.
"""
from .network import (CONFIG_C, Network, Server, bstest, clamp_words, clock_s, config, kwtatest,  # noqa: F401
                      load_stim, multi_train, noisy_cue, noisy_cue_seed, stimuli)

__all__ = ["Network", "Server", "config", "CONFIG_C", "stimuli", "load_stim", "bstest", "multi_train", "clock_s",
           "clamp_words", "noisy_cue", "noisy_cue_seed", "kwtatest"]
