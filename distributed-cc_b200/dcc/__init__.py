"""dcc -- B200 (sm_100a) implementation of Distributed-CC's triples/quadruples
hot path.  Importing the package loads libdcc_b200.so and fails loudly when it
has not been built."""
from . import _lib  # noqa: F401  (loads the CUDA library or raises ImportError)

__all__ = ["_lib"]
