"""VTK ImageData output of device fields (glide/io.py:20-202).

``write_vti`` writes one snapshot in the VTK XML ImageData format the
reference writes: point data as Float32 arrays in a raw appended block, each
preceded by its UInt32 byte count, scalar fields as one component and vector
fields as stacked components, an optional ``TimeValue`` field, rows flipped to
VTK's upward y by default.  ``VTIWriter`` writes a numbered series
(``<base>_<step:04d>.vti``) and a ``.pvd`` collection for ParaView.

Unlike the reference, the writer does not stop the host for the file: each
``write_step`` copies the fields device -> pinned host on a side stream
(after an event on the producing stream; later work on the producing stream
waits only for that copy, so the snapshot holds the values at the call) and a
background thread waits for the copy and writes the file, so the host keeps
launching while the disk write runs.  ``flush`` (or ``close``) waits for
pending files.
HDF5 output (glide/io.py:205-282) needs h5py, which this image does not have.
"""
from __future__ import annotations

import queue
import threading
import xml.etree.ElementTree as ET
from pathlib import Path
from xml.dom import minidom

import numpy as np
import torch


def _to_host32(x):
    if isinstance(x, torch.Tensor):
        return x.detach().to("cpu", torch.float32).numpy()
    return np.asarray(x, dtype=np.float32)


def _vti_bytes(fields, dx, dy, origin, time_value, flip_y):
    """fields: ordered (name, [component arrays]) with host float32 arrays."""
    prep = []
    for name, comps in fields:
        comps = [np.flip(c, axis=0) if flip_y else c for c in comps]
        prep.append((name, comps))
    ny, nx = prep[0][1][0].shape
    root = ET.Element("VTKFile", type="ImageData", version="1.0", byte_order="LittleEndian",
                      header_type="UInt32")
    img = ET.SubElement(root, "ImageData", WholeExtent=f"0 {nx - 1} 0 {ny - 1} 0 0",
                        Origin=f"{origin[0]} {origin[1]} 0", Spacing=f"{dx} {dy} 1.0")
    piece = ET.SubElement(img, "Piece", Extent=f"0 {nx - 1} 0 {ny - 1} 0 0")
    if time_value is not None:
        fd = ET.SubElement(piece, "FieldData")
        tv = ET.SubElement(fd, "DataArray", type="Float32", Name="TimeValue", NumberOfComponents="1",
                           format="ascii")
        tv.text = f"{float(time_value)}"
    attrs = {}
    scalars = [n for n, c in prep if len(c) == 1]
    vectors3 = [n for n, c in prep if len(c) == 3]
    if scalars:
        attrs["Scalars"] = scalars[0]
    if vectors3:
        attrs["Vectors"] = vectors3[0]
    pd = ET.SubElement(piece, "PointData", **attrs)
    blobs, offset = [], 0
    for name, comps in prep:
        arr = comps[0] if len(comps) == 1 else np.stack(comps, axis=-1)
        raw = np.ascontiguousarray(arr, dtype="<f4").tobytes()
        ET.SubElement(pd, "DataArray", type="Float32", Name=name, NumberOfComponents=str(len(comps)),
                      format="appended", offset=str(offset))
        blobs.append(raw)
        offset += 4 + len(raw)
    ET.SubElement(root, "AppendedData", encoding="raw")
    head = ET.tostring(root, encoding="unicode")
    head = head.replace('<AppendedData encoding="raw" />', "")
    head = head.replace("</VTKFile>", "")
    body = bytearray(('<?xml version="1.0"?>\n' + head + '<AppendedData encoding="raw">\n_').encode())
    for raw in blobs:
        body += np.uint32(len(raw)).tobytes() + raw
    body += b"\n</AppendedData>\n</VTKFile>\n"
    return bytes(body)


def _fields(data):
    out = []
    for name, value in data.items():
        comps = value if isinstance(value, (list, tuple)) else [value]
        out.append((name, comps))
    return out


def write_vti(filename, data, dx, dy=None, origin=(0.0, 0.0), time_value=None, flip_y=True):
    """One VTI snapshot (glide/io.py:20-137); ``data`` maps names to a 2-D array
    (scalar) or a list of 2-D arrays (vector), device tensors or host arrays."""
    dy = dx if dy is None else dy
    path = Path(filename)
    path.parent.mkdir(parents=True, exist_ok=True)
    host = [(n, [_to_host32(c) for c in comps]) for n, comps in _fields(data)]
    path.write_bytes(_vti_bytes(host, dx, dy, origin, time_value, flip_y))
    return path


def read_vti(filename):
    """Fields of a VTI file written by ``write_vti`` as {name: array (ny, nx[, ncomp])},
    rows in the file's (VTK) order, plus the time value when present."""
    blob = Path(filename).read_bytes()
    start = blob.index(b'<AppendedData encoding="raw">')
    xml_head = blob[:start].decode() + "</VTKFile>"
    root = ET.fromstring(xml_head.split("?>", 1)[1])
    img = root.find("ImageData")
    x0, x1, y0, y1, _, _ = (int(t) for t in img.get("WholeExtent").split())
    nx, ny = x1 - x0 + 1, y1 - y0 + 1
    data_start = blob.index(b"_", start) + 1
    out = {}
    for da in root.iter("DataArray"):
        if da.get("format") == "ascii":
            out[da.get("Name")] = float(da.text)
            continue
        off = data_start + int(da.get("offset"))
        n = int(np.frombuffer(blob, dtype="<u4", count=1, offset=off)[0])
        arr = np.frombuffer(blob, dtype="<f4", count=n // 4, offset=off + 4)
        nc = int(da.get("NumberOfComponents"))
        out[da.get("Name")] = arr.reshape(ny, nx) if nc == 1 else arr.reshape(ny, nx, nc)
    return out


class VTIWriter:
    """Numbered VTI series plus a PVD collection (glide/io.py:140-202), written
    asynchronously from device buffers."""

    def __init__(self, out_dir, base="output", dx=1.0, dy=None, origin=(0.0, 0.0), flip_y=True):
        self.out_dir = Path(out_dir)
        self.out_dir.mkdir(parents=True, exist_ok=True)
        self.base = base
        self.dx, self.dy = float(dx), float(dx if dy is None else dy)
        self.origin = origin
        self.flip_y = flip_y
        self.records = []
        self._queue = queue.Queue()
        self._errors = []
        self._stream = None
        self._thread = threading.Thread(target=self._worker, daemon=True)
        self._thread.start()

    def _snapshot(self, data):
        """Start device -> pinned host copies of every field after the producing
        stream's current work; returns the host buffers and the copy event."""
        fields = _fields(data)
        on_gpu = any(isinstance(c, torch.Tensor) and c.is_cuda for _, comps in fields for c in comps)
        if not on_gpu:
            return [(n, [_to_host32(c) for c in comps]) for n, comps in fields], None
        if self._stream is None:
            self._stream = torch.cuda.Stream()
        producer = torch.cuda.current_stream()
        ready = torch.cuda.Event()
        ready.record(producer)
        host = []
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(ready)
            for name, comps in fields:
                bufs = []
                for c in comps:
                    src = c.detach()
                    src32 = src if src.dtype == torch.float32 else src.to(torch.float32)
                    # the source must outlive the copy: the side stream is told it uses it
                    src32.record_stream(self._stream)
                    dst = torch.empty(src32.shape, dtype=torch.float32, pin_memory=True)
                    dst.copy_(src32, non_blocking=True)
                    bufs.append(dst)
                host.append((name, bufs))
            done = torch.cuda.Event()
            done.record(self._stream)
        # later work on the producing stream may overwrite the fields: it waits
        # for the (short) device -> host copy, the host does not
        producer.wait_event(done)
        return host, done

    def _worker(self):
        while True:
            item = self._queue.get()
            if item is None:
                self._queue.task_done()
                return
            path, host, done, time_value = item
            try:
                if done is not None:
                    done.synchronize()
                arrays = [(n, [b.numpy() if isinstance(b, torch.Tensor) else b for b in bufs]) for n, bufs in host]
                path.write_bytes(_vti_bytes(arrays, self.dx, self.dy, self.origin, time_value, self.flip_y))
            except Exception as e:  # reported by flush()
                self._errors.append((path, e))
            finally:
                self._queue.task_done()

    def write_step(self, step_idx, time_value, data):
        """Queue one numbered snapshot; returns its path (written in the background)."""
        fname = f"{self.base}_{step_idx:04d}.vti"
        path = self.out_dir / fname
        host, done = self._snapshot(data)
        self._queue.put((path, host, done, time_value))
        self.records.append((float(time_value), fname))
        return path

    def flush(self):
        """Wait until every queued snapshot is on disk; raises the first write error."""
        self._queue.join()
        if self._errors:
            path, err = self._errors[0]
            raise RuntimeError(f"writing {path} failed: {err}") from err

    def write_pvd(self, pvd_name=None):
        """Write the PVD collection of the snapshots so far (after flushing them)."""
        self.flush()
        pvd_name = pvd_name or f"{self.base}.pvd"
        root = ET.Element("VTKFile", type="Collection", version="0.1", byte_order="LittleEndian")
        coll = ET.SubElement(root, "Collection")
        for t, fname in self.records:
            ET.SubElement(coll, "DataSet", timestep=str(t), group="", part="0", file=fname)
        text = minidom.parseString(ET.tostring(root)).toprettyxml(indent="  ")
        path = self.out_dir / pvd_name
        path.write_text(text)
        return path

    def close(self):
        self.flush()
        self._queue.put(None)
        self._thread.join(timeout=60)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
