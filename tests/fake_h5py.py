"""An in-memory stand-in for the part of h5py an HDF5 layout writer uses
(test infrastructure: h5py is not installed here).

`File(path, mode)` keeps a tree of groups and datasets in a module-level
registry keyed by path, so a test can open what a writer wrote.  Datasets
record shape, dtype, chunks and compression settings and hold their data in a
numpy array; strings are stored as Python str in object arrays.
`describe(file)` returns the layout and a digest of every dataset's
contents, the form the golden layout fixture stores.
"""
from __future__ import annotations

import hashlib

import numpy as np

_FILES: dict = {}


class _StringDtype:
    def __repr__(self):
        return "string_dtype"


_STR = _StringDtype()


def string_dtype(encoding: str = "utf-8", length=None):
    return _STR


def _is_str(dtype) -> bool:
    return dtype is _STR


class Dataset:
    def __init__(self, name, shape, dtype, data, chunks, compression, compression_opts):
        self.name = name
        self.chunks = None if chunks is None else tuple(int(c) for c in chunks)
        self.compression = compression
        self.compression_opts = compression_opts
        self.is_string = _is_str(dtype) or (isinstance(data, (str, bytes)) and dtype is None)
        if self.is_string:
            if data is not None and shape is None:
                self.data = np.array(data if isinstance(data, str) else data.decode(), dtype=object)
            else:
                self.data = np.full(tuple(shape), "", dtype=object)
            self.dtype = "str"
        else:
            if data is not None:
                arr = np.asarray(data) if dtype is None else np.asarray(data, dtype=dtype)
                self.data = arr.copy()
            else:
                self.data = np.zeros(tuple(shape), dtype=dtype)
            self.dtype = self.data.dtype.str
        self.shape = tuple(self.data.shape)

    def __setitem__(self, key, value):
        if self.is_string:
            self.data[key] = value if isinstance(value, str) else bytes(value).decode()
        else:
            self.data[key] = np.asarray(value)

    def __getitem__(self, key):
        v = self.data[key]
        if self.is_string and isinstance(v, str):
            return v.encode()
        return v


class Group:
    def __init__(self):
        self.items: dict = {}

    def _resolve(self, path: str):
        node = self
        for part in [p for p in path.split("/") if p]:
            node = node.items[part]
        return node

    def __getitem__(self, path):
        return self._resolve(path)

    def __contains__(self, path):
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False

    def create_group(self, name: str) -> "Group":
        if name in self.items:
            raise ValueError(f"group {name} exists")
        g = Group()
        self.items[name] = g
        return g

    def create_dataset(self, name, shape=None, dtype=None, data=None, chunks=None, compression=None,
                       compression_opts=None, **kw):
        if name in self.items:
            raise ValueError(f"dataset {name} exists")
        ds = Dataset(name, shape, dtype, data, chunks, compression, compression_opts)
        self.items[name] = ds
        return ds


class File(Group):
    def __init__(self, path, mode: str = "r"):
        super().__init__()
        self.path = str(path)
        self.mode = mode
        if mode == "w":
            _FILES[self.path] = self
        else:
            self.items = _FILES[self.path].items
        self.flushes = 0

    def flush(self):
        self.flushes += 1

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def describe(node: Group, prefix: str = "") -> dict:
    """{path: {shape, dtype, chunks, compression, compression_opts, digest}}
    for every dataset under node (strings digested as UTF-8 text)."""
    out = {}
    for name, item in sorted(node.items.items()):
        path = f"{prefix}/{name}"
        if isinstance(item, Group):
            out.update(describe(item, path))
            continue
        if item.is_string:
            text = "\x00".join(str(x) for x in np.ravel(item.data))
            digest = hashlib.sha256(text.encode()).hexdigest()
        else:
            digest = hashlib.sha256(np.ascontiguousarray(item.data).tobytes()).hexdigest()
        out[path] = {"shape": list(item.shape), "dtype": item.dtype,
                     "chunks": None if item.chunks is None else list(item.chunks),
                     "compression": item.compression, "compression_opts": item.compression_opts,
                     "digest": digest}
    return out
