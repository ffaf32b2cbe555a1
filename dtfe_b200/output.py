"""Field files in the reference's binary output format (outputFileType 101).

writeOutputData (src/input_output.cc:216-275) writes every selected field to
its own file, named after the output name plus a per-field suffix, through
writeBinaryFile (src/io/binary_io.cc:185-216): the raw floats of the
Quantities vector (cells x components), native byte order, no header.
``write_fields`` does the same for host arrays (numpy) through
``dtfe_write_binary`` and for device tensors (torch, CUDA) through a handle's
``dtfe_gpu_write_binary_dev``, which streams them to the file through pinned
buffers without a host copy of its own.
"""
from __future__ import annotations

import numpy as np

from . import _native as N


def suffix(field: str, averaged: bool = False) -> str | None:
    """writeOutputData's file suffix of `field` (".den", ".a_den", ...);
    None for a field without a file (the unaveraged velocity std)."""
    s = N.host().dtfe_field_suffix(N.FIELD_SLOTS[field], 1 if averaged else 0)
    return s.decode() if s else None


def write_binary(path: str, data) -> None:
    """Raw floats of a host array (any shape, float32) to `path`."""
    a = np.ascontiguousarray(data, np.float32)
    N.check(N.host().dtfe_write_binary(path.encode(), a.ctypes.data, a.nbytes))


def write_fields(base: str, fields: dict, averaged: bool = False, device=None) -> list[str]:
    """Writes each field of `fields` (name -> array or CUDA tensor, rows x
    components) to `base` + its suffix, in the field-slot order
    writeOutputData uses; device tensors need `device` (a DeviceDTFE whose
    stream orders the copies).  Returns the paths written."""
    paths = []
    for name in sorted(fields, key=lambda f: N.FIELD_SLOTS[f]):
        sfx = suffix(name, averaged)
        if sfx is None:
            raise ValueError(f"the reference writes no file for {name} (averaged={averaged})")
        path = base + sfx
        a = fields[name]
        if hasattr(a, "is_cuda") and a.is_cuda:
            if device is None:
                raise ValueError("device tensors need the DeviceDTFE handle that produced them")
            device.write_binary_dev(path, a)
        else:
            write_binary(path, a)
        paths.append(path)
    return paths
