"""naer_b200 — B200-native (sm_100a) spiking-network simulation step.

The package is a thin host layer over the CUDA library
``libnaer_b200.so`` (C ABI: include/naer/naer_capi.h).  ``Network`` mirrors
the reference's C++ model-building API; ``spec`` holds the declarative
network description and the benchmark workloads; ``forms`` has the batched
(``Batch``) and served (``Server``) forms.
"""
from ._capi import NaerError, load  # noqa: F401
from .network import Connection, Network, NeuronType, Population  # noqa: F401
from .forms import Batch, Server  # noqa: F401

__all__ = ["Network", "NeuronType", "Population", "Connection", "NaerError", "load", "Batch", "Server"]
