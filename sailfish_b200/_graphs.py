"""
CUDA-graph capture shared by the solvers. Captures run one at a time (a
process-wide lock) in thread-local capture mode, so that host threads
driving other streams (the batched adjoint) may keep launching and
synchronising their own streams while a capture is open.
"""

import contextlib
import threading

_LOCK = threading.Lock()


@contextlib.contextmanager
def capture(graph, stream):
    import torch

    with _LOCK:
        with torch.cuda.graph(graph, stream=stream, capture_error_mode="thread_local"):
            yield
