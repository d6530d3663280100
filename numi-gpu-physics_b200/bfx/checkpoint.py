"""Checkpoint archive: a directory with a JSON manifest and raw data files,
each named in the manifest with its byte count and SHA-256 digest.

The layout follows the reference's CheckpointArchive
(Sources/BirdFlowMetal/CheckpointArchive.swift:23-160): `manifest.json`
(schema, configuration, bird, step, time, body, load, and per file the byte
count and digest), `populations` and `solid-mask`, written into a temporary
sibling directory that replaces the destination only once complete.  Two
differences:

* the data files are raw: the reference compresses them with LZFSE, an
  Apple-only codec;
* a third file, `restart-state.raw`, holds the library's exact restart state
  (bfx_save_state: populations in their storage format, both mask buffers, the
  wall field and the device state), so a restore resumes bit for bit.  The
  populations file is the canonical FP32 field the reference stores, and a
  restore checks it against the restored simulation.
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import uuid

SCHEMA_VERSION = 1
MANIFEST = "manifest.json"
POPULATIONS = "populations.raw"
SOLID_MASK = "solid-mask.raw"
RESTART_STATE = "restart-state.raw"
# manifest key prefix of each data file
FILE_KEYS = {POPULATIONS: "population", SOLID_MASK: "solidMask", RESTART_STATE: "restartState"}


class CheckpointError(Exception):
    """An archive that cannot be read back: missing file, unsupported schema,
    empty numerical state, size or digest mismatch."""


def sha256(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


def write_archive(destination: str, manifest: dict, files: dict) -> None:
    """Writes `files` (name -> bytes) and the manifest (with schema, byte
    counts and digests added) into `destination`, replacing it atomically."""
    destination = os.path.abspath(destination)
    parent = os.path.dirname(destination)
    os.makedirs(parent, exist_ok=True)
    temporary = os.path.join(parent, f".{os.path.basename(destination)}-{uuid.uuid4().hex}")
    os.makedirs(temporary)
    try:
        m = dict(manifest)
        m["schema"] = SCHEMA_VERSION
        for name, data in files.items():
            key = FILE_KEYS.get(name, name)
            m[f"{key}Bytes"] = len(data)
            m[f"{key}SHA256"] = sha256(data)
            with open(os.path.join(temporary, name), "wb") as fh:
                fh.write(data)
        with open(os.path.join(temporary, MANIFEST), "w") as fh:
            json.dump(m, fh, indent=2, sort_keys=True)
        if os.path.exists(destination):
            shutil.rmtree(destination)
        os.replace(temporary, destination)
    except BaseException:
        shutil.rmtree(temporary, ignore_errors=True)
        raise


def read_archive(source: str, names=(POPULATIONS, SOLID_MASK, RESTART_STATE)):
    """Reads and verifies an archive: (manifest, {name: bytes})."""
    try:
        with open(os.path.join(source, MANIFEST)) as fh:
            manifest = json.load(fh)
    except (OSError, ValueError) as e:
        raise CheckpointError(f"unreadable manifest: {e}") from e
    if manifest.get("schema") != SCHEMA_VERSION:
        raise CheckpointError(f"unsupported schema {manifest.get('schema')!r}")
    files = {}
    for name in names:
        key = FILE_KEYS.get(name, name)
        size = manifest.get(f"{key}Bytes")
        digest = manifest.get(f"{key}SHA256")
        if not isinstance(size, int) or size <= 0 or not isinstance(digest, str):
            raise CheckpointError(f"{name}: missing or empty in the manifest")
        try:
            with open(os.path.join(source, name), "rb") as fh:
                data = fh.read()
        except OSError as e:
            raise CheckpointError(f"{name}: {e}") from e
        if len(data) != size:
            raise CheckpointError(f"{name}: {len(data)} bytes, manifest says {size}")
        if sha256(data) != digest:
            raise CheckpointError(f"{name}: checksum mismatch")
        files[name] = data
    return manifest, files


def struct_from_dict(cls, d: dict):
    """The inverse of struct_dict: a ctypes structure of type `cls` filled from
    plain values (nested structures and arrays included); fields absent from
    `d` keep their zero value."""
    s = cls()
    for name, _ in cls._fields_:
        if name.startswith("_") or name not in d:
            continue
        value = d[name]
        cur = getattr(s, name)
        if hasattr(cur, "_fields_"):
            setattr(s, name, struct_from_dict(type(cur), value))
        elif hasattr(cur, "__len__") and not isinstance(cur, (bytes, str)):
            for i, e in enumerate(value):
                if hasattr(cur[i], "_fields_"):
                    cur[i] = struct_from_dict(type(cur[i]), e)
                elif hasattr(cur[i], "__len__"):
                    cur[i][:] = list(e)
                else:
                    cur[i] = e
        else:
            setattr(s, name, value)
    return s


def struct_dict(s) -> dict:
    """A ctypes structure as plain JSON values (arrays as lists)."""
    out = {}
    for name, _ in s._fields_:
        if name.startswith("_"):
            continue
        v = getattr(s, name)
        if hasattr(v, "_fields_"):
            v = struct_dict(v)
        elif hasattr(v, "__len__") and not isinstance(v, (bytes, str)):
            v = [struct_dict(e) if hasattr(e, "_fields_") else (list(e) if hasattr(e, "__len__") else e) for e in v]
        elif isinstance(v, bytes):
            continue
        out[name] = v
    return out
