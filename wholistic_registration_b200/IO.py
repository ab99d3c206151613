"""Output formats of the registration pipeline (utils/IO.py:737-1033).

The reference writes registered volumes with tifffile (ImageJ hyperstack
TIFF, ``saveTiff_new`` / ``write_volume_as_ome_tiff``; multi-page BigTIFF,
``saveTiff``) and zarr (``saveZarr`` / ``saveZarr_fast``).  Neither library
is part of this package's dependencies, so the formats are written here
directly:

* TIFF: little-endian, one uncompressed strip per page, classic TIFF below
  4 GiB and BigTIFF above (or on request), uint8 / uint16 / float32 /
  (for ``saveTiff``) any numeric dtype; ImageJ hyperstacks carry the ImageJ
  description (images, channels, slices, frames, hyperstack, mode, and the
  caller's metadata keys) and the resolution tags, with pages in T, Z, C
  order as ImageJ reads them.
* zarr (format 2): a directory store (or a zip archive with
  ``single_file``) holding a group with the arrays "membrane", "calcium" and
  "reference" and the configuration in the group attributes; chunks are
  compressed with zlib (the reference's default Blosc codec needs numcodecs).

ND2 input (``readND2Frame``) needs Nikon's SDK reader and stays outside this
package.  Registered volumes on the GPU are copied to the host once per
write.
"""

from __future__ import annotations

import json
import os
import struct
import zipfile
import zlib

import numpy as np

__all__ = ["saveTiff", "saveTiff_new", "readTiff", "write_volume_as_ome_tiff",
           "write_multichannel_volume_as_ome_tiff", "read_reg_tiff", "saveZarr", "saveZarr_fast", "readZarr"]

# ---------------------------------------------------------------------------
# TIFF
# ---------------------------------------------------------------------------

_SAMPLE_FORMAT = {"u": 1, "i": 2, "f": 3}
_TYPE_SHORT, _TYPE_LONG, _TYPE_RATIONAL, _TYPE_ASCII, _TYPE_LONG8 = 3, 4, 5, 2, 16


def _host(a):
    if hasattr(a, "detach"):          # torch tensors (CUDA or CPU)
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def _rational(v):
    """(numerator, denominator) of a positive float, 32-bit each."""
    v = float(v)
    den = 1
    while abs(v * den - round(v * den)) > 1e-9 * max(1.0, v * den) and den < 1_000_000:
        den *= 10
    return int(round(v * den)) & 0xFFFFFFFF, den


class _TiffWriter:
    """Pages appended one at a time: the page data, then its IFD."""

    def __init__(self, path, bigtiff):
        self.f = open(path, "wb")
        self.big = bigtiff
        if bigtiff:
            self.f.write(b"II" + struct.pack("<HHHQ", 43, 8, 0, 0))
            self.link = 8          # where the next IFD offset goes
        else:
            self.f.write(b"II" + struct.pack("<HI", 42, 0))
            self.link = 4

    def _pos(self):
        return self.f.tell()

    def _align(self):
        if self._pos() % 2:
            self.f.write(b"\0")

    def page(self, img, description=None, resolution=None, photometric=1):
        img = np.ascontiguousarray(img)
        if img.dtype.byteorder == ">" or (img.dtype.byteorder == "=" and not np.little_endian):
            img = img.astype(img.dtype.newbyteorder("<"))
        h, w = img.shape[:2]
        spp = img.shape[2] if img.ndim == 3 else 1
        self._align()
        data_off = self._pos()
        self.f.write(img.tobytes())
        entries = []

        def add(tag, typ, values):
            if typ == _TYPE_ASCII:
                raw = values
                count = len(raw)
            else:
                fmt = {_TYPE_SHORT: "H", _TYPE_LONG: "I", _TYPE_RATIONAL: "II", _TYPE_LONG8: "Q"}[typ]
                flat = [x for v in values for x in (v if isinstance(v, tuple) else (v,))]
                raw = struct.pack("<" + fmt[0] * len(flat), *flat)
                count = len(values)
            entries.append([tag, typ, count, raw])

        add(254, _TYPE_LONG, [0])
        add(256, _TYPE_LONG, [w])
        add(257, _TYPE_LONG, [h])
        add(258, _TYPE_SHORT, [img.dtype.itemsize * 8] * spp)
        add(259, _TYPE_SHORT, [1])
        add(262, _TYPE_SHORT, [photometric])
        if description is not None:
            add(270, _TYPE_ASCII, description.encode("utf-8") + b"\0")
        add(273, _TYPE_LONG8 if self.big else _TYPE_LONG, [data_off])
        add(277, _TYPE_SHORT, [spp])
        add(278, _TYPE_LONG, [h])
        add(279, _TYPE_LONG8 if self.big else _TYPE_LONG, [img.nbytes])
        if resolution is not None:
            add(282, _TYPE_RATIONAL, [_rational(resolution[0])])
            add(283, _TYPE_RATIONAL, [_rational(resolution[1])])
            add(296, _TYPE_SHORT, [1])
        if spp > 1:
            add(284, _TYPE_SHORT, [1])
        add(339, _TYPE_SHORT, [_SAMPLE_FORMAT[img.dtype.kind]] * spp)
        entries.sort(key=lambda e: e[0])
        inline = 8 if self.big else 4
        # out-of-line values first, then the IFD
        for e in entries:
            if len(e[3]) > inline:
                self._align()
                off = self._pos()
                self.f.write(e[3])
                e[3] = struct.pack("<Q" if self.big else "<I", off)
            else:
                e[3] = e[3].ljust(inline, b"\0")
        self._align()
        ifd = self._pos()
        if self.big:
            self.f.write(struct.pack("<Q", len(entries)))
            for tag, typ, count, raw in entries:
                self.f.write(struct.pack("<HHQ", tag, typ, count) + raw)
            nxt = self._pos()
            self.f.write(struct.pack("<Q", 0))
        else:
            self.f.write(struct.pack("<H", len(entries)))
            for tag, typ, count, raw in entries:
                self.f.write(struct.pack("<HHI", tag, typ, count) + raw)
            nxt = self._pos()
            self.f.write(struct.pack("<I", 0))
        end = self._pos()
        self.f.seek(self.link)
        self.f.write(struct.pack("<Q" if self.big else "<I", ifd))
        self.f.seek(end)
        self.link = nxt

    def close(self):
        self.f.close()


def _write_pages(path, pages, nbytes, description=None, resolution=None, bigtiff=None, photometric=1):
    big = bool(bigtiff) if bigtiff is not None else nbytes > 2 ** 32 - 2 ** 25
    w = _TiffWriter(path, big)
    try:
        for i, p in enumerate(pages):
            w.page(p, description if i == 0 else None, resolution, photometric)
    finally:
        w.close()


def _read_pages(path):
    """(pages, first description) of a TIFF written as above (uncompressed
    strips, any number per page, classic or BigTIFF)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:2] != b"II":
        raise ValueError(f"{path}: only little-endian TIFF is read")
    magic = struct.unpack_from("<H", buf, 2)[0]
    big = magic == 43
    if magic not in (42, 43):
        raise ValueError(f"{path}: not a TIFF file")
    off = struct.unpack_from("<Q", buf, 8)[0] if big else struct.unpack_from("<I", buf, 4)[0]
    sizes = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 16: 8}
    fmts = {1: "B", 2: "B", 3: "H", 4: "I", 5: "I", 16: "Q"}
    pages, desc = [], None
    while off:
        n = struct.unpack_from("<Q" if big else "<H", buf, off)[0]
        p = off + (8 if big else 2)
        tags = {}
        for _ in range(n):
            if big:
                tag, typ, count = struct.unpack_from("<HHQ", buf, p)
                vp, inline = p + 12, 8
                p += 20
            else:
                tag, typ, count = struct.unpack_from("<HHI", buf, p)
                vp, inline = p + 8, 4
                p += 12
            size = sizes.get(typ, 1) * count
            at = vp if size <= inline else struct.unpack_from("<Q" if big else "<I", buf, vp)[0]
            if typ == 2:
                tags[tag] = buf[at:at + count].rstrip(b"\0").decode("utf-8", "replace")
            else:
                k = count * (2 if typ == 5 else 1)
                tags[tag] = list(struct.unpack_from("<" + fmts[typ] * k, buf, at))
        off = struct.unpack_from("<Q" if big else "<I", buf, p)[0]
        if desc is None and 270 in tags:
            desc = tags[270]
        w, h = tags[256][0], tags[257][0]
        bits = tags[258][0]
        spp = tags.get(277, [1])[0]
        kind = {1: "u", 2: "i", 3: "f"}[tags.get(339, [1])[0]]
        if tags.get(259, [1])[0] != 1:
            raise ValueError(f"{path}: compressed TIFF pages are not read")
        dt = np.dtype(f"<{kind}{bits // 8}")
        raw = b"".join(buf[o:o + c] for o, c in zip(tags[273], tags[279]))
        img = np.frombuffer(raw, dtype=dt, count=w * h * spp).reshape((h, w, spp) if spp > 1 else (h, w))
        pages.append(img)
    return pages, desc


def _imagej_description(shape_tzcyx, metadata):
    t, z, c = shape_tzcyx[:3]
    lines = ["ImageJ=1.11a", f"images={t * z * c}"]
    if c > 1:
        lines.append(f"channels={c}")
    if z > 1:
        lines.append(f"slices={z}")
    if t > 1:
        lines.append(f"frames={t}")
    if c > 1 or z > 1 or t > 1:
        lines.append("hyperstack=true")
    lines.append("mode=grayscale")
    for k, v in (metadata or {}).items():
        lines.append(f"{k}={json.dumps(list(v)) if isinstance(v, tuple) else v}")
    lines.append("loop=false")
    return "\n".join(lines) + "\n"


def _imagej_shape(desc, n, page_shape):
    """Hyperstack shape of an ImageJ description (singleton axes dropped, as
    tifffile returns the series)."""
    keys = {}
    for line in (desc or "").splitlines():
        if "=" in line:
            k, v = line.split("=", 1)
            keys[k.strip()] = v.strip()
    if "ImageJ" not in keys:
        return (n,) + page_shape if n > 1 else page_shape
    t, z, c = int(keys.get("frames", 1)), int(keys.get("slices", 1)), int(keys.get("channels", 1))
    if t * z * c != n:
        return (n,) + page_shape
    return tuple(d for d in (t, z, c) if d > 1) + page_shape


def saveTiff(image_list, config_path, save_path):
    """utils/IO.py:737-768: frames as a multi-page BigTIFF whose description
    is the TOML configuration serialised as JSON."""
    import toml

    config_str = json.dumps(toml.load(config_path), ensure_ascii=False)
    for i, img in enumerate(image_list):
        if not isinstance(_host(img), np.ndarray):
            raise ValueError(f"element{i} is not a image")
    stack = np.asarray([_host(i) for i in image_list])
    rgb = stack.ndim == 4 and stack.shape[-1] in (3, 4)
    pages = [stack[k] for k in range(stack.shape[0])] if stack.ndim in (3, 4) and (stack.ndim == 3 or rgb) \
        else list(stack.reshape((-1,) + stack.shape[-2:]))
    _write_pages(save_path, pages, stack.nbytes, description=config_str, bigtiff=True,
                 photometric=2 if rgb else 1)


def saveTiff_new(image, save_path, config_path=None, metadata=None, verbose=True):
    """utils/IO.py:771-810: a 5-D (T, Z, C, Y, X) image (or one 2-D plane) as
    an ImageJ hyperstack TIFF with the spacing as resolution and in the
    description, plus the configuration path ("config") when given."""
    image = _host(image)
    if image.ndim == 2:
        image = image[None, None, None, :, :]
    if image.ndim != 5:
        raise ValueError("All saved should be 5D (TZCYX)")
    if image.dtype == bool:
        image = image.astype(np.uint8)
    if image.dtype not in (np.uint8, np.uint16, np.float32):
        image = image.astype(np.float32)
    if metadata is not None:
        spacing_x, spacing_y = metadata["spacing_x"], metadata["spacing_y"]
        metadata = {**metadata, "data_shape": image.shape}
    else:
        spacing_x = spacing_y = 1
        metadata = {"spacing_x": 1, "spacing_y": 1, "data_shape": image.shape}
    if config_path is not None:
        metadata = {**metadata, "config": config_path}
    if verbose:
        print(f"Saving TIFF file to {save_path}")
        print(f"  - shape: {image.shape}")
        print(f"  - spacing: {spacing_x}, {spacing_y}")
        if config_path is not None:
            print(f"  - config: {config_path}")
    t, z, c, y, x = image.shape
    pages = (image[ti, zi, ci] for ti in range(t) for zi in range(z) for ci in range(c))
    _write_pages(save_path, pages, image.nbytes, description=_imagej_description(image.shape, metadata),
                 resolution=(1.0 / spacing_x, 1.0 / spacing_y))


def readTiff(tiff_path):
    """utils/IO.py:933-939: (image array, first page's description).  ImageJ
    hyperstacks come back with their singleton axes dropped."""
    pages, desc = _read_pages(tiff_path)
    arr = np.stack(pages)
    return arr.reshape(_imagej_shape(desc, len(pages), pages[0].shape)), desc


def _frame_tag(frame_idx):
    if isinstance(frame_idx, (int, np.integer)):
        return f"{int(frame_idx):06d}"
    if not isinstance(frame_idx, str):
        raise TypeError("frame_idx must be int or string")
    parts = frame_idx.replace("-", "~").replace("_", "~").split("~")
    try:
        if len(parts) == 1:
            return f"{int(parts[0]):06d}"
        if len(parts) == 2:
            return f"{int(parts[0]):06d}_{int(parts[1]):06d}"
        if len(parts) == 5:
            a, b, c, d = int(parts[0]), int(parts[1]), int(parts[3]), int(parts[4])
            return f"{a:04d}~{b:04d}_vs_{c:04d}~{d:04d}"
    except ValueError:
        raise ValueError(f"Invalid frame_idx string: {frame_idx}") from None
    raise ValueError(f"Invalid frame_idx format: {frame_idx}")


def write_volume_as_ome_tiff(volume, out_dir, ch_idx, frame_idx, configPath, spacing_x=1.0, spacing_y=1.0):
    """utils/IO.py:942-993: a (Z, Y, X) or (Y, X) volume as
    ``out_dir/vol_<ch_idx>_<frame tag>.tif`` (ImageJ hyperstack, 1 x Z x 1 x Y x X)."""
    volume = _host(volume)
    tag = _frame_tag(frame_idx)
    if volume.ndim == 2:
        zvol = volume[np.newaxis]
    elif volume.ndim == 3:
        zvol = volume
    else:
        raise ValueError("volume must be 2D or 3D (Z,Y,X)")
    img5d = zvol[np.newaxis, :, np.newaxis, :, :]
    os.makedirs(out_dir, exist_ok=True)
    fname = os.path.join(out_dir, f"vol_{ch_idx}_{tag}.tif")
    metadata = {"spacing_x": spacing_x, "spacing_y": spacing_y, "data_shape": img5d.shape}
    saveTiff_new(img5d, fname, config_path=configPath, metadata=metadata, verbose=False)
    return fname


def write_multichannel_volume_as_ome_tiff(volume, out_dir, frame_idx, configPath=None, label=None, spacing_x=1.0,
                                          spacing_y=1.0):
    """utils/IO.py:996-1024: c volumes (Z, Y, X) as one (1, Z, c, Y, X) ImageJ
    hyperstack ``out_dir/vol_<label>_<frame>.tif``."""
    processed = []
    for v in volume:
        v = _host(v)
        if v.ndim == 2:
            v = v[np.newaxis]
        if v.dtype == bool:
            v = v.astype(np.uint8)
        elif v.dtype not in (np.uint8, np.float32):
            v = v.astype(np.float32)
        processed.append(v)
    img5d = np.transpose(np.stack(processed, axis=0)[np.newaxis], (0, 2, 1, 3, 4))
    fname = os.path.join(out_dir, f"vol_{label}_{int(frame_idx):06d}.tif")
    metadata = {"spacing_x": spacing_x, "spacing_y": spacing_y, "data_shape": img5d.shape}
    saveTiff_new(img5d, fname, config_path=configPath, metadata=metadata, verbose=False)


def read_reg_tiff(folder, frame_idx, ch_idx):
    """utils/IO.py:1027-1033: the (Z, Y, X) volume ``vol_ch<ch>_<frame>.tif``."""
    fname = os.path.join(folder, f"vol_ch{ch_idx}_{frame_idx:06d}.tif")
    if not os.path.exists(fname):
        raise FileNotFoundError(f"Cannot find {fname}")
    return readTiff(fname)[0]


# ---------------------------------------------------------------------------
# zarr (format 2)
# ---------------------------------------------------------------------------

_ZLIB_DEFAULT = {"id": "zlib", "level": 1}


class _DirStore:
    def __init__(self, path):
        self.path = path
        if os.path.isdir(path):
            import shutil

            shutil.rmtree(path)
        os.makedirs(path)

    def put(self, key, data):
        full = os.path.join(self.path, *key.split("/"))
        os.makedirs(os.path.dirname(full), exist_ok=True)
        with open(full, "wb") as fh:
            fh.write(data)

    def close(self):
        pass


class _ZipStore:
    def __init__(self, path):
        self.z = zipfile.ZipFile(path, "w", compression=zipfile.ZIP_STORED, allowZip64=True)

    def put(self, key, data):
        self.z.writestr(key, data)

    def close(self):
        self.z.close()


def _zarr_array(store, name, data, chunks, compressor):
    """One zarr v2 array: .zarray metadata and C-order chunks named "i.j.k",
    edge chunks padded with the fill value 0 to the full chunk shape."""
    data = np.ascontiguousarray(data)
    if chunks is None:
        chunks = data.shape
    chunks = tuple(int(min(c, s)) if s > 0 else int(c) for c, s in zip(chunks, data.shape))
    chunks = chunks + data.shape[len(chunks):]
    meta = {"zarr_format": 2, "shape": list(data.shape), "chunks": list(chunks), "dtype": data.dtype.str,
            "compressor": compressor, "fill_value": 0, "order": "C", "filters": None}
    store.put(f"{name}/.zarray", json.dumps(meta, indent=4, sort_keys=True).encode())
    grid = [-(-s // c) for s, c in zip(data.shape, chunks)]
    for idx in np.ndindex(*grid):
        sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunks, data.shape))
        block = data[sl]
        if block.shape != chunks:
            full = np.zeros(chunks, dtype=data.dtype)
            full[tuple(slice(0, b) for b in block.shape)] = block
            block = full
        raw = np.ascontiguousarray(block).tobytes()
        if compressor is not None:
            raw = zlib.compress(raw, int(compressor.get("level", 1)))
        store.put(f"{name}/" + ".".join(str(i) for i in idx), raw)


def _save_zarr(mem_data, ca_data, reference, config_path, save_path, chunks, compressor, single_file):
    import toml

    config_str = json.dumps(toml.load(config_path), ensure_ascii=False)
    mem = np.asarray(_host(mem_data), dtype=np.float32)
    ca = np.asarray(_host(ca_data), dtype=np.float32)
    ref = np.asarray(_host(reference), dtype=np.float32)
    if compressor is not None and compressor.get("id") != "zlib":
        raise ValueError("compressor must be None (raw chunks) or {'id': 'zlib', 'level': n}")
    store = _ZipStore(save_path + ".zip") if single_file else _DirStore(save_path)
    try:
        store.put(".zgroup", json.dumps({"zarr_format": 2}).encode())
        store.put(".zattrs", json.dumps({"config": config_str}, ensure_ascii=False).encode("utf-8"))
        _zarr_array(store, "membrane", mem, chunks, compressor)
        _zarr_array(store, "calcium", ca, chunks, compressor)
        _zarr_array(store, "reference", ref, None, compressor)
    finally:
        store.close()
    print(f"Saved Zarr dataset at {save_path}")
    print(f"  - membrane: {mem.shape}")
    print(f"  - calcium : {ca.shape}")
    print(f"  - reference: {ref.shape}")


def saveZarr(mem_data, ca_data, reference, config_path, save_path, chunks=(1, 512, 512)):
    """utils/IO.py:813-853: membrane, calcium and reference as float32 arrays
    of one zarr group (directory store), the configuration (TOML serialised
    as JSON) in its "config" attribute; zlib-compressed chunks."""
    _save_zarr(mem_data, ca_data, reference, config_path, save_path, chunks, dict(_ZLIB_DEFAULT), False)


def saveZarr_fast(mem_data, ca_data, reference, config_path, save_path, chunks=(16, 512, 512), compressor=None,
                  single_file=False):
    """utils/IO.py:856-930: saveZarr with larger chunks, a chosen compressor
    (None: zlib level 1; ``{"id": "zlib", "level": n}``; ``"raw"``: none) and
    optionally one zip archive (``save_path + ".zip"``)."""
    comp = None if compressor == "raw" else (dict(_ZLIB_DEFAULT) if compressor is None else compressor)
    _save_zarr(mem_data, ca_data, reference, config_path, save_path, chunks, comp, single_file)


def readZarr(path):
    """{name: array} and the group attributes of a store written by
    saveZarr / saveZarr_fast (directory or ``.zip``)."""
    if path.endswith(".zip"):
        z = zipfile.ZipFile(path)
        get = z.read
        names = z.namelist()
    else:
        def get(key):
            with open(os.path.join(path, *key.split("/")), "rb") as fh:
                return fh.read()
        names = []
        for root, _, files in os.walk(path):
            names += [os.path.relpath(os.path.join(root, f), path).replace(os.sep, "/") for f in files]
    attrs = json.loads(get(".zattrs")) if ".zattrs" in names else {}
    out = {}
    for key in names:
        if not key.endswith("/.zarray"):
            continue
        name = key[: -len("/.zarray")]
        meta = json.loads(get(key))
        shape, chunks, dt = tuple(meta["shape"]), tuple(meta["chunks"]), np.dtype(meta["dtype"])
        arr = np.zeros(shape, dtype=dt)
        grid = [-(-s // c) for s, c in zip(shape, chunks)]
        for idx in np.ndindex(*grid):
            raw = get(f"{name}/" + ".".join(str(i) for i in idx))
            if meta["compressor"] is not None:
                raw = zlib.decompress(raw)
            block = np.frombuffer(raw, dtype=dt).reshape(chunks)
            sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunks, shape))
            arr[sl] = block[tuple(slice(0, x.stop - x.start) for x in sl)]
        out[name] = arr
    return out, attrs
