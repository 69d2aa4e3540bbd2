"""Corpus I/O: a code file or host array streamed into device memory.

``load_codes(source, space)`` returns a CUDA uint8 tensor ``[n, code_size]``
holding the codes of ``source``: a ``.npy`` file, a raw file of packed codes
(the reference's layout, ``n * code_size_bytes()`` bytes), or any host buffer.
The file is memory-mapped and copied in chunks through two pinned staging
buffers, so reading chunk i+1 from the page cache overlaps the host-to-device
copy of chunk i; the corpus never has to fit in host memory at once.
"""
from __future__ import annotations

import os

import numpy as np


def _source_bytes(source, cs):
    if isinstance(source, (str, os.PathLike)):
        path = os.fspath(source)
        if path.endswith(".npy"):
            arr = np.load(path, mmap_mode="r")
            if arr.dtype != np.uint8:
                raise ValueError("codes must be uint8")
        else:
            arr = np.memmap(path, dtype=np.uint8, mode="r")
    else:
        mv = memoryview(source)
        if mv.itemsize != 1:
            raise ValueError("codes must be uint8")
        arr = np.asarray(mv).view(np.uint8)
    flat = arr.reshape(-1)
    if flat.size % cs != 0:
        raise ValueError("codes size not a multiple of code_size_bytes")
    return flat


def load_codes(source, space, device=None, chunk_bytes=256 << 20):
    """Codes of `source` (path or host buffer) as a CUDA uint8 tensor [n, cs]
    on `device` (default: the space's device)."""
    import torch

    cs = space.code_size_bytes()
    flat = _source_bytes(source, cs)
    n = flat.size // cs
    dev = torch.device("cuda", space.device() if device is None else int(device))
    out = torch.empty((n, cs), dtype=torch.uint8, device=dev)
    if n == 0:
        return out
    per = max(1, int(chunk_bytes) // cs) * cs  # whole codes per chunk
    per = min(per, flat.size)
    stream = torch.cuda.Stream(dev)
    stage = [torch.empty(per, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    done = [None, None]
    dst = out.view(-1)
    for k, off in enumerate(range(0, flat.size, per)):
        b = k & 1
        nb = min(per, flat.size - off)
        if done[b] is not None:
            done[b].synchronize()  # the copy that last read this staging buffer
        stage[b].numpy()[:nb] = flat[off:off + nb]
        with torch.cuda.stream(stream):
            dst[off:off + nb].copy_(stage[b][:nb], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        done[b] = ev
    stream.synchronize()
    torch.cuda.current_stream(dev).wait_stream(stream)
    return out
