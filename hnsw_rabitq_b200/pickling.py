"""The reference's pickled state of an ``hnswlib.Index`` and its saved-index
file, each built from the other.

``hnswlib.Index.__getstate__`` returns ``(getIndexParams(),)``
(python_bindings/bindings.cpp:465-482, 1001-1008): a dict of scalar
parameters plus ``getAnnData()`` (bindings.cpp:351-462), which copies the
level-0 block, the upper-level link lists, ``element_levels_`` and the label
map.  ``HierarchicalNSW::saveIndex`` (hnswlib/hnswalg.h:685-712) writes the same
fields in a fixed layout: a header, the level-0 block of the
``cur_element_count`` elements, then per element its upper-level list size
(uint32) and the list.  The GPU index loads that file layout, so a pickled
state is turned back into file bytes (``state_to_file_bytes``) and a loaded
file into a state (``file_bytes_to_state``).
"""
from __future__ import annotations

import struct

import numpy as np

SER_VERSION = 1  # bindings.cpp:148
# offsetLevel0_, max_elements_, cur_element_count, size_data_per_element_,
# label_offset_, offsetData_ (size_t); maxlevel_ (int); enterpoint_node_
# (uint32); maxM_, maxM0_, M_ (size_t); mult_ (double); ef_construction_
_HEADER = struct.Struct("<QQQQQQiIQQQdQ")


def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a)).view(np.uint8).reshape(-1)


def state_to_file_bytes(d: dict) -> bytes:
    """saveIndex's file for the index described by a getIndexParams dict."""
    if not d.get("index_inited", True):
        raise RuntimeError("the state holds no index (index_inited is false)")
    cur = int(d["cur_element_count"])
    size_data = int(d["size_data_per_element"])
    size_links = int(d["size_links_per_element"])
    head = _HEADER.pack(int(d["offset_level0"]), int(d["max_elements"]), cur, size_data, int(d["label_offset"]),
                        int(d["offset_data"]), int(d["max_level"]), int(d["enterpoint_node"]), int(d["max_M"]),
                        int(d["max_M0"]), int(d["M"]), float(d["mult"]), int(d["ef_construction"]))
    level0 = _u8(d["data_level0"])[: cur * size_data]
    if level0.size != cur * size_data:
        raise RuntimeError("data_level0 is shorter than cur_element_count elements")
    levels = np.asarray(d["element_levels"], np.int64)[:cur]
    links = _u8(d["link_lists"])
    parts = [head, level0.tobytes()]
    off = 0
    for lev in levels:
        n = size_links * int(lev) if lev > 0 else 0
        parts.append(struct.pack("<I", n))
        if n:
            if off + n > links.size:
                raise RuntimeError("link_lists is shorter than element_levels requires")
            parts.append(links[off:off + n].tobytes())
        off += n
    return b"".join(parts)


def file_bytes_to_state(buf: bytes, space: str, dim: int, ef: int, num_threads: int = -1, seed: int = 100) -> dict:
    """The getIndexParams dict of the index stored in a saveIndex file.
    The label map lists elements in internal-id order (the reference lists it
    in its hash map's order)."""
    (off0, max_el, cur, size_data, label_off, data_off, maxlevel, ep, maxM, maxM0, M, mult,
     efc) = _HEADER.unpack_from(buf, 0)
    pos = _HEADER.size
    level0 = np.frombuffer(buf, np.uint8, cur * size_data, pos)
    pos += cur * size_data
    size_links = maxM * 4 + 4
    levels = np.zeros(max_el, np.int32)
    chunks = []
    for i in range(cur):
        (n,) = struct.unpack_from("<I", buf, pos)
        pos += 4
        if n:
            levels[i] = n // size_links
            chunks.append(buf[pos:pos + n])
            pos += n
    if pos != len(buf):
        raise RuntimeError("Index seems to be corrupted or unsupported")
    rec = level0.reshape(cur, size_data) if cur else level0.reshape(0, max(size_data, 1))
    labels = rec[:, label_off:label_off + 8].copy().view(np.uint64).reshape(-1)
    deleted = (rec[:, off0 + 2] & 1) != 0 if cur else np.zeros(0, bool)
    return {
        "ser_version": SER_VERSION, "space": space, "dim": int(dim), "index_inited": True, "ep_added": cur > 0,
        "normalize": space == "cosine", "num_threads": int(num_threads), "seed": int(seed),
        "offset_level0": off0, "max_elements": max_el, "cur_element_count": cur, "size_data_per_element": size_data,
        "label_offset": label_off, "offset_data": data_off, "max_level": maxlevel, "enterpoint_node": ep,
        "max_M": maxM, "max_M0": maxM0, "M": M, "mult": mult, "ef_construction": efc, "ef": int(ef),
        "has_deletions": bool(deleted.any()), "size_links_per_element": size_links, "allow_replace_deleted": False,
        "label_lookup_external": labels, "label_lookup_internal": np.arange(cur, dtype=np.uint32),
        "element_levels": levels, "data_level0": level0.view(np.int8).copy(),
        "link_lists": np.frombuffer(b"".join(chunks), np.int8).copy(),
    }


def set_delete_marks(buf: bytes, deleted_labels: set, undeleted_labels: set) -> bytes:
    """A copy of a saveIndex file with the delete mark (bit 0 of the third
    byte of each element's level-0 list header, hnswalg.h:872-935) set for
    `deleted_labels` and cleared for `undeleted_labels`."""
    if not deleted_labels and not undeleted_labels:
        return buf
    (off0, _, cur, size_data, label_off, *_rest) = _HEADER.unpack_from(buf, 0)
    out = bytearray(buf)
    base = _HEADER.size
    for i in range(cur):
        r = base + i * size_data
        (lab,) = struct.unpack_from("<Q", out, r + label_off)
        if lab in deleted_labels:
            out[r + off0 + 2] |= 1
        elif lab in undeleted_labels:
            out[r + off0 + 2] &= 0xFE
    return bytes(out)


def items_from_file(buf: bytes, ids, dim: int, elem_dtype=np.float32) -> np.ndarray:
    """getDataByLabel (hnswalg.h:825-846) for each label of `ids`, read from a
    saveIndex file: rows of `dim` elements.  A label that is absent or marked
    deleted raises "Label not found", as the reference does."""
    (off0, _, cur, size_data, label_off, data_off, *_rest) = _HEADER.unpack_from(buf, 0)
    rec = np.frombuffer(buf, np.uint8, cur * size_data, _HEADER.size).reshape(cur, size_data)
    labels = rec[:, label_off:label_off + 8].copy().view(np.uint64).reshape(-1)
    where = {int(v): i for i, v in enumerate(labels.tolist())}
    width = dim * np.dtype(elem_dtype).itemsize
    out = np.empty((len(ids), dim), np.float32)
    for r, lab in enumerate(ids):
        i = where.get(int(lab))
        if i is None or rec[i, off0 + 2] & 1:
            raise RuntimeError("Label not found")
        out[r] = rec[i, data_off:data_off + width].copy().view(elem_dtype)
    return out


def with_max_elements(buf: bytes, max_elements: int) -> bytes:
    """A copy of a saveIndex file whose header records another max_elements_
    (what resizeIndex changes, hnswalg.h:633-656)."""
    out = bytearray(buf)
    struct.pack_into("<Q", out, 8, int(max_elements))
    return bytes(out)


# BruteforceSearch::saveIndex / loadIndex (hnswlib/bruteforce.h:128-161):
# maxelements_, size_per_element_, cur_element_count (size_t), then
# maxelements_ records of (vector, label).
_BF_HEADER = struct.Struct("<QQQ")


def bf_file_to_rows(buf: bytes, dim: int):
    """(max_elements, rows [cur, dim] float32, labels [cur] uint64) of a
    brute-force index file."""
    maxel, size_per, cur = _BF_HEADER.unpack_from(buf, 0)
    if size_per != dim * 4 + 8 or len(buf) < _BF_HEADER.size + maxel * size_per or cur > maxel:
        raise RuntimeError("Index seems to be corrupted or unsupported")
    rec = np.frombuffer(buf, np.uint8, cur * size_per, _BF_HEADER.size).reshape(cur, size_per)
    rows = rec[:, :dim * 4].copy().view(np.float32).reshape(cur, dim)
    labels = rec[:, dim * 4:].copy().view(np.uint64).reshape(cur)
    return int(maxel), rows, labels


def bf_rows_to_file(rows: np.ndarray, labels: np.ndarray, max_elements: int, dim: int) -> bytes:
    """The brute-force index file of these rows (records beyond the current
    count are zero; the reference writes whatever its buffer holds there)."""
    cur = rows.shape[0]
    size_per = dim * 4 + 8
    rec = np.zeros((max(int(max_elements), cur), size_per), np.uint8)
    if cur:
        rec[:cur, :dim * 4] = np.ascontiguousarray(rows, np.float32).view(np.uint8).reshape(cur, dim * 4)
        rec[:cur, dim * 4:] = np.ascontiguousarray(labels, np.uint64).view(np.uint8).reshape(cur, 8)
    return _BF_HEADER.pack(rec.shape[0], size_per, cur) + rec.tobytes()


class RecordReader:
    """Reads single elements of a saveIndex file (a path, read by seeking, or
    the file's bytes) without loading the whole level-0 block."""

    def __init__(self, src):
        self._bytes = src if isinstance(src, (bytes, bytearray)) else None
        self._f = None if self._bytes is not None else open(src, "rb")
        head = self._read(0, _HEADER.size)
        (self.off0, _, self.cur, self.size_data, self.label_off, self.data_off, *_rest) = _HEADER.unpack(head)

    def _read(self, pos: int, n: int) -> bytes:
        if self._bytes is not None:
            return bytes(self._bytes[pos:pos + n])
        self._f.seek(pos)
        return self._f.read(n)

    def _rec(self, i: int) -> int:
        if not 0 <= i < self.cur:
            raise IndexError(i)
        return _HEADER.size + i * self.size_data

    def deleted(self, i: int) -> bool:
        return (self._read(self._rec(i) + self.off0 + 2, 1)[0] & 1) != 0

    def vector(self, i: int, dim: int, elem_dtype=np.float32) -> np.ndarray:
        w = dim * np.dtype(elem_dtype).itemsize
        return np.frombuffer(self._read(self._rec(i) + self.data_off, w), elem_dtype).astype(np.float32)

    def close(self):
        if self._f is not None:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _fma32(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """float32 fused multiply-add, correctly rounded: the float64 product of
    two float32 values is exact, TwoSum gives the exact error of adding c, and
    that error decides the one case float64 rounding can get wrong (a sum
    exactly halfway between two float32 values)."""
    p = a.astype(np.float64) * b.astype(np.float64)
    c64 = c.astype(np.float64)
    t = p + c64
    bb = t - p
    err = (p - (t - bb)) + (c64 - bb)
    r = t.astype(np.float32)
    up = np.nextafter(r, np.float32(np.inf))
    dn = np.nextafter(r, np.float32(-np.inf))
    r64 = r.astype(np.float64)
    r = np.where((t == (r64 + up.astype(np.float64)) / 2) & (err > 0), up, r)
    r = np.where((t == (r64 + dn.astype(np.float64)) / 2) & (err < 0), dn, r)
    return r.astype(np.float32)


def normalize_rows(x: np.ndarray) -> np.ndarray:
    """The reference's normalize_vector (bindings.cpp:241-248) over rows, in
    the arithmetic of its optimised build (the one the GPU's norm_scale
    reproduces): the squares of the first dim - dim % 4 elements are rounded
    and added in order, the last dim % 4 are fused multiply-adds, then
    x * (1 / (sqrt(norm) + 1e-30)), all in float32."""
    x = np.ascontiguousarray(x, np.float32)
    n, dim = x.shape
    n4 = dim & ~3
    s = np.zeros(n, np.float32)
    for i in range(n4):
        s = (s + (x[:, i] * x[:, i]).astype(np.float32)).astype(np.float32)
    for i in range(n4, dim):
        s = _fma32(x[:, i], x[:, i], s)
    sc = (np.float32(1.0) / (np.sqrt(s) + np.float32(1e-30))).astype(np.float32)
    return (x * sc[:, None]).astype(np.float32)
