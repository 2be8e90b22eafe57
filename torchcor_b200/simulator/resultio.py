"""Result files written while the steps run.

``Vm.pt`` of a solve is the stack of snapshot frames saved with ``torch.save``
(torchcor/simulator/monodomain.py:207-208).  Written after the last step, it adds
a device-to-host copy of every frame and a file write of the whole stack to the
end of the solve.  ``StreamedTensorFile`` produces the same file while the
frames are being computed:

* ``torch.save`` first writes a template of the tensor (same shape and dtype) to
  the path, so every record of the archive (the pickle, the version records, the
  storage record) is laid out by torch itself;
* each row's bytes then go to their place in the storage record (``pwrite``) as
  soon as the row is on the host, in row order;
* the zip format keeps a CRC-32 of every record: ``torch.save`` writes each record
  with a data descriptor (general-purpose flag bit 3; the local header's CRC is 0)
  and repeats the CRC in the central directory.  The CRC of the storage record is
  accumulated over the rows and written into both places at the end.

``torch.load`` reads the result as it reads ``torch.save``'s own file, and
``zipfile``'s CRC check passes.  ``FrameWriter`` drives one such file from the
device: a thread of its own copies each snapshot frame to pinned host memory on
its own stream, once the compute stream has produced it, and writes it.
"""
from __future__ import annotations

import os
import struct
import threading
import time
import zipfile
import zlib
from pathlib import Path

import torch

_LOCAL = 0x04034B50
_CENTRAL = 0x02014B50
_DESCRIPTOR = 0x08074B50


class StreamedTensorFile:
    """``torch.save`` of a contiguous tensor of ``shape`` and ``dtype`` at ``path``,
    whose rows (along the first dimension) are supplied one at a time, in order."""

    def __init__(self, path, shape, dtype=torch.float32):
        self.path = os.fspath(path)
        self.shape = tuple(int(s) for s in shape)
        if not self.shape:
            raise ValueError("StreamedTensorFile needs at least one dimension")
        self.dtype = dtype
        self.n_rows = self.shape[0]
        row = 1
        for s in self.shape[1:]:
            row *= s
        self.row_bytes = row * torch.empty((), dtype=dtype).element_size()
        torch.save(torch.empty(self.shape, dtype=dtype), self.path)
        self._locate()
        self._fd = os.open(self.path, os.O_RDWR)
        self._crc = 0
        self.rows_written = 0

    def _locate(self):
        with zipfile.ZipFile(self.path) as z:
            recs = [i for i in z.infolist() if i.filename.endswith("/data/0")]
            if len(recs) != 1:
                raise RuntimeError(f"{self.path}: expected one storage record, found {len(recs)}")
            info = recs[0]
            start_dir = z.start_dir
        with open(self.path, "rb") as f:
            f.seek(info.header_offset)
            sig, _, flags, comp, _, _, _, _, _, nl, el = struct.unpack("<IHHHHHIIIHH", f.read(30))
            if sig != _LOCAL or comp != 0:
                raise RuntimeError(f"{self.path}: storage record is not stored uncompressed")
            self._data = info.header_offset + 30 + nl + el
            if info.file_size != self.n_rows * self.row_bytes:
                raise RuntimeError(f"{self.path}: storage record holds {info.file_size} bytes, "
                                   f"expected {self.n_rows * self.row_bytes}")
            # where the record's CRC lives: its data descriptor (flag bit 3; the
            # descriptor's signature is optional) or its local header
            self._crc_at = []
            if flags & 0x8:
                f.seek(self._data + info.file_size)
                (w,) = struct.unpack("<I", f.read(4))
                self._crc_at.append(self._data + info.file_size + (4 if w == _DESCRIPTOR else 0))
            else:
                self._crc_at.append(info.header_offset + 14)
            # and its central-directory entry
            f.seek(start_dir)
            name = info.orig_filename.encode("utf-8")
            while True:
                pos = f.tell()
                head = f.read(46)
                if len(head) < 46 or struct.unpack("<I", head[:4])[0] != _CENTRAL:
                    raise RuntimeError(f"{self.path}: storage record missing from the central directory")
                nl, el, cl = struct.unpack("<HHH", head[28:34])
                if f.read(nl) == name:
                    self._crc_at.append(pos + 16)
                    break
                f.seek(el + cl, os.SEEK_CUR)

    def write_row(self, i, data):
        """Row ``i`` (must be the next one) from a C-contiguous host buffer of
        ``row_bytes`` bytes (numpy array, memoryview, bytes)."""
        if i != self.rows_written:
            raise ValueError(f"rows must arrive in order: got {i}, expected {self.rows_written}")
        mv = memoryview(data).cast("B")
        if mv.nbytes != self.row_bytes:
            raise ValueError(f"row {i} has {mv.nbytes} bytes, expected {self.row_bytes}")
        off = self._data + i * self.row_bytes
        done = 0
        while done < mv.nbytes:
            done += os.pwrite(self._fd, mv[done:], off + done)
        self._crc = zlib.crc32(mv, self._crc)
        self.rows_written += 1

    def close(self):
        """Write the CRC once every row is in; the file is then complete."""
        if self._fd is None:
            return
        try:
            if self.rows_written != self.n_rows:
                raise RuntimeError(f"{self.path}: {self.rows_written} of {self.n_rows} rows written")
            crc = struct.pack("<I", self._crc & 0xFFFFFFFF)
            for at in self._crc_at:
                os.pwrite(self._fd, crc, at)
        finally:
            os.close(self._fd)
            self._fd = None

    def abandon(self):
        """Close without completing (the caller removes or overwrites the file)."""
        if self._fd is not None:
            os.close(self._fd)
            self._fd = None


class FrameWriter:
    """Writes ``frames`` (a device tensor [F, ...], row f = snapshot frame f) to
    ``path`` as ``torch.save(frames.cpu())`` would, while the compute stream is still
    producing later frames.  The caller reports progress with ``produced(k, event)``
    (frames 0..k-1 are complete once ``event`` has completed) and ends with
    ``finish(event)`` after the last frame; ``abort()`` on an error path."""

    def __init__(self, path, frames: torch.Tensor):
        if not frames.is_cuda or not frames.is_contiguous():
            raise ValueError("FrameWriter needs a contiguous CUDA tensor")
        self.path = Path(path)
        self.frames = frames
        self.device = frames.device
        self.n = frames.shape[0]
        self._cv = threading.Condition()
        self._marks = []          # (frames complete, event), in order
        self._abort = False
        self._error = None
        self.times = {}       # perf_counter marks of the writer thread: start, template, done
        row = frames[0]
        self._pinned = [torch.empty(row.shape, dtype=row.dtype, pin_memory=True) for _ in range(2)]
        self._stream = torch.cuda.Stream(self.device)
        self._thread = threading.Thread(target=self._run, name="torchcor-vm-writer", daemon=True)
        self._thread.start()

    def produced(self, count, event):
        with self._cv:
            self._marks.append((int(count), event))
            self._cv.notify()

    def _next_mark(self, after):
        with self._cv:
            while not self._abort and not any(c > after for c, _ in self._marks):
                self._cv.wait()
            if self._abort:
                return None
            c, ev = next((c, ev) for c, ev in self._marks if c > after)
            self._marks = [m for m in self._marks if m[0] > c]
            return c, ev

    def _run(self):
        out = None
        try:
            self.times["start"] = time.perf_counter()
            out = StreamedTensorFile(self.path, tuple(self.frames.shape), self.frames.dtype)
            self.times["template"] = time.perf_counter()
            with torch.cuda.device(self.device):
                ready = 0        # frames 0..ready-1 are complete once this stream has waited their event
                f = 0            # next frame to copy to the host
                pending = None   # (frame, pinned slot, copy event): copied, not yet written
                while f < self.n or pending is not None:
                    nxt = None
                    if f < self.n:
                        if f >= ready and pending is None:
                            m = self._next_mark(f)          # blocks until frame f is produced
                            if m is None:
                                return                       # aborted
                            self._stream.wait_event(m[1])
                            ready = m[0]
                        if f < ready:
                            # frame f's copy overlaps the write of the previous frame (other slot)
                            slot = self._pinned[f % 2]
                            with torch.cuda.stream(self._stream):
                                slot.copy_(self.frames[f], non_blocking=True)
                            ev = torch.cuda.Event()
                            ev.record(self._stream)
                            nxt = (f, slot, ev)
                            f += 1
                    if pending is not None:
                        pf, ps, pe = pending
                        pe.synchronize()
                        out.write_row(pf, ps.numpy())
                    pending = nxt
            out.close()
            out = None
            self.times["done"] = time.perf_counter()
        except BaseException as e:      # reported by finish()
            self._error = e
        finally:
            if out is not None:
                out.abandon()

    def finish(self, event):
        """The last frame is complete once ``event`` has; waits for the file."""
        self.produced(self.n, event)
        self._thread.join()
        if self._error is not None:
            raise RuntimeError(f"writing {self.path} failed") from self._error
        if self._abort:
            raise RuntimeError(f"writing {self.path} was aborted")

    def abort(self):
        with self._cv:
            self._abort = True
            self._cv.notify()
        self._thread.join()
