"""What a run writes: measurement rows, array snapshots and run metadata, in
the reference's formats (crates/virial/src/data.rs, manifest.rs).

When recording into a directory, rows go to `measurements.csv`, snapshots to
`<name>.npy` and metadata to `run.json`. Numbers are written in their shortest
exact form, as the reference writes them (Rust's `{:?}` for f64): reading a
value back gives exactly the f64 that was written, and the text is the
reference's, byte for byte.
"""

import math
import os
import struct

import numpy as np


def exact(v):
    """Shortest decimal that reads back as exactly `v`, spelled as Rust's
    `{:?}` spells an f64 (data.rs:120-125): `1.0`, `0.1`, `-0.0`, `1e-5`,
    `6.02214076e23`, `inf`, `NaN`."""
    v = float(v)
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    text = repr(v)  # shortest round trip; scientific below 1e-4 and from 1e16, as Rust
    if "e" in text:
        mantissa, exponent = text.split("e")
        if mantissa.endswith(".0"):
            mantissa = mantissa[:-2]
        sign = "-" if exponent.startswith("-") else ""
        digits = exponent.lstrip("+-").lstrip("0") or "0"
        return f"{mantissa}e{sign}{digits}"
    return text


def npy(shape, data):
    """NumPy `.npy` (format 1.0) bytes for a little-endian f64 array, header
    padded to 64 bytes (data.rs:127-146)."""
    shape = [int(d) for d in shape]
    values = np.ascontiguousarray(data, dtype="<f8").reshape(-1)
    if int(np.prod(shape)) != values.size:
        raise ValueError("shape doesn't match data")
    dims = [str(d) for d in shape]
    shape_text = f"({dims[0]},)" if len(dims) == 1 else "(" + ", ".join(dims) + ")"
    header = "{'descr': '<f8', 'fortran_order': False, 'shape': " + shape_text + ", }"
    unpadded = 10 + len(header) + 1
    header += " " * ((64 - unpadded % 64) % 64) + "\n"
    return (b"\x93NUMPY\x01\x00" + struct.pack("<H", len(header)) + header.encode("ascii")
            + values.tobytes())


def json_string(s):
    """A JSON string literal, escaped as the reference escapes it
    (data.rs:148-162)."""
    out = ['"']
    for c in str(s):
        if c == '"':
            out.append('\\"')
        elif c == "\\":
            out.append("\\\\")
        elif c == "\n":
            out.append("\\n")
        elif ord(c) < 0x20:
            out.append(f"\\u{ord(c):04x}")
        else:
            out.append(c)
    out.append('"')
    return "".join(out)


def fnv1a(data):
    """FNV-1a 64-bit hash (manifest.rs:6-14), for checking that reruns are
    identical."""
    h = 0xCBF29CE484222325
    for b in bytes(data):
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


class DataLog:
    """Where a run's data goes (data.rs:14-118): measurement rows (the first
    row sets the columns), settings and facts for `run.json`, and snapshots
    written as `.npy` when recording into a directory."""

    def __init__(self, directory=None):
        self.directory = directory
        self.columns = []
        self.rows = []
        self.meta_entries = []
        if directory is not None:
            os.makedirs(directory, exist_ok=True)

    def is_recording(self):
        return self.directory is not None

    def row(self, values):
        """Adds a row: a sequence of (name, value) pairs, the same names in
        the same order every time."""
        names = [name for name, _ in values]
        if not self.columns:
            self.columns = names
        elif names != self.columns:
            raise ValueError("measurement columns changed between rows")
        self.rows.append([float(v) for _, v in values])

    def meta(self, key, value):
        """Records a setting or fact about the run (the last value for a key
        wins, in first-seen order)."""
        for entry in self.meta_entries:
            if entry[0] == key:
                entry[1] = str(value)
                return
        self.meta_entries.append([key, str(value)])

    def snapshot(self, name, shape, data):
        """Writes `data` (row-major, `shape`) to `<name>.npy` when recording."""
        payload = npy(shape, data)
        if self.directory is not None:
            with open(os.path.join(self.directory, f"{name}.npy"), "wb") as f:
                f.write(payload)

    def csv(self):
        lines = [",".join(self.columns)]
        lines += [",".join(exact(v) for v in row) for row in self.rows]
        return "\n".join(lines) + "\n"

    def write(self, manifest=None):
        """Writes `measurements.csv` and, given a Manifest, `run.json`."""
        if self.directory is None:
            return
        with open(os.path.join(self.directory, "measurements.csv"), "w") as f:
            f.write(self.csv())
        if manifest is not None:
            with open(os.path.join(self.directory, "run.json"), "w") as f:
                f.write(manifest.json(self))


class Manifest:
    """The facts `run.json` records (manifest.rs:16-67). `settings` is a list
    of (key, value) pairs, written sorted."""

    def __init__(self, title, gpu, version, commit=None, uncommitted_changes=None, width=0,
                 height=0, fps=0, frames=0, seconds=0.0, settings=()):
        self.title, self.gpu, self.version = title, gpu, version
        self.commit, self.uncommitted_changes = commit, uncommitted_changes
        self.width, self.height, self.fps, self.frames = width, height, fps, frames
        self.seconds = seconds
        self.settings = [(str(k), str(v)) for k, v in settings]

    def json(self, data):
        fields = [
            ("scene", json_string(self.title)),
            ("virial_version", json_string(self.version)),
            ("git_commit", "null" if self.commit is None else json_string(self.commit)),
            ("git_uncommitted_changes", "null" if self.uncommitted_changes is None
             else ("true" if self.uncommitted_changes else "false")),
            ("gpu", json_string(self.gpu)),
            ("width", str(self.width)),
            ("height", str(self.height)),
            ("fps", str(self.fps)),
            ("frames", str(self.frames)),
            ("render_seconds", f"{self.seconds:.3f}"),
            ("settings", "{" + ", ".join(f"{json_string(k)}: {json_string(v)}"
                                         for k, v in sorted(self.settings)) + "}"),
        ]
        out = "{\n" + "".join(f"  {json_string(k)}: {v},\n" for k, v in fields)
        scene = ", ".join(f"{json_string(k)}: {json_string(v)}" for k, v in data.meta_entries)
        return out + f'  "scene_meta": {{{scene}}}\n}}\n'
