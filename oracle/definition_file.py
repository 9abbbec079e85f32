"""ORACLE / TEST INFRASTRUCTURE ONLY.

A structure definition as a file, so that a process can hand the CPU
checkers a definition without loading the product library itself.
`save` (run where the product library builds the definition) writes the raw
bytes of every array of a swb_structure_definition into one .npz; `load`
rebuilds the same C struct from those bytes with ctypes alone.  The
reference arm of bench.py uses it: a child process generates the wing and
saves it, and the timed process loads it and steps the reference build
(oracle/_ref) on it, with no product library mapped.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from simwing_b200 import abi

# (count field, pointer field, element type) of the top-level arrays
_ARRAYS = (("node_count", "nodes", abi.NodeDef), ("triangle_count", "triangles", abi.TriangleDef),
           ("constraint_count", "constraints", abi.ConstraintDef), ("membrane_count", "membranes", abi.MembraneDef),
           ("dihedral_count", "dihedrals", abi.DihedralDef))
_SUSPENSION_ARRAYS = (("attachment_count", "attachments", abi.SuspensionAttachment),
                      ("junction_count", "junctions", abi.SuspensionJunction),
                      ("harness_count", "harness_points", abi.PilotHarness),
                      ("segment_count", "segments", abi.SuspensionSegment))


def _bytes_of(pointer, count, ctype) -> np.ndarray:
    if not count:
        return np.zeros(0, dtype=np.uint8)
    return np.frombuffer(C.string_at(pointer, count * C.sizeof(ctype)), dtype=np.uint8).copy()


def save(definition, path: str) -> None:
    """Writes `definition` (anything with a `.view` StructureDefinition)."""
    v = definition.view
    out = {}
    for count, field, ctype in _ARRAYS:
        out[field] = _bytes_of(getattr(v, field), getattr(v, count), ctype)
    if v.fabric_self_contact:
        out["fabric_self_contact"] = _bytes_of(v.fabric_self_contact, 1, abi.FabricContactDef)
    if v.suspension:
        s = v.suspension.contents
        out["suspension"] = np.frombuffer(bytes(s), dtype=np.uint8).copy()
        for count, field, ctype in _SUSPENSION_ARRAYS:
            out["suspension_" + field] = _bytes_of(getattr(s, field), getattr(s, count), ctype)
    np.savez(path, **out)


class FileDefinition:
    """A StructureDefinition over buffers read from a file: `.pointer` and
    `.view` as the product's Definition offers them."""

    def __init__(self, path: str):
        data = np.load(path)
        self._keep = []
        v = abi.StructureDefinition()
        for count, field, ctype in _ARRAYS:
            setattr(v, count, 0)
            self._attach(v, count, field, ctype, data[field])
        if "fabric_self_contact" in data:
            fc = abi.FabricContactDef.from_buffer_copy(data["fabric_self_contact"].tobytes())
            self._keep.append(fc)
            v.fabric_self_contact = C.pointer(fc)
        if "suspension" in data:
            s = abi.SuspensionDef.from_buffer_copy(data["suspension"].tobytes())
            for count, field, ctype in _SUSPENSION_ARRAYS:
                self._attach(s, count, field, ctype, data["suspension_" + field])
            self._keep.append(s)
            v.suspension = C.pointer(s)
        self.view = v

    def _attach(self, owner, count, field, ctype, raw):
        n = raw.size // C.sizeof(ctype)
        if n * C.sizeof(ctype) != raw.size:
            raise ValueError(f"definition file: {field} is not a whole number of records")
        arr = (ctype * max(n, 1)).from_buffer_copy(raw.tobytes() if n else bytes(C.sizeof(ctype)))
        self._keep.append(arr)
        setattr(owner, count, n)
        setattr(owner, field, C.cast(arr, C.POINTER(ctype)) if n else C.POINTER(ctype)())

    @property
    def pointer(self):
        return C.pointer(self.view)

    @property
    def node_count(self) -> int:
        return int(self.view.node_count)
