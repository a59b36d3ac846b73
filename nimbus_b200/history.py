"""History output of resident runs: frames copied out of HBM with cell-centred
velocities and written as the reference's npy history.

The reference exports a frame (src/core/runtime/headless_runtime.cpp:2440-2625)
by recreating <outdir>/step_NNNNNN, staging cell-centre u, v, w
(interpolate_*_face_to_center) and writing each active core field as
<name>.npy with npy::write_3d, either at once or from its asynchronous
writer's thread (src/core/output/output_writer.cpp:1330-1350).

Here a frame is enqueued on the run's own stream (nimbus_cuda_history_snapshot
for a ResidentRun, nimbus_cuda_engine_history_async for an engine member: one
centring launch, one copy for the velocities and one per scalar field into a
pinned image), and a writer thread waits for that frame's event and writes the
files with nimbus_history_write.  The steps enqueued after a frame overlap both its copy
and its file writes; the writer blocks new frames only when every pinned
image is still in flight.
"""
from __future__ import annotations

import queue
import shutil
import threading
from pathlib import Path

import numpy as np
import torch

from . import cuda


def frame_dir(outdir, index: int) -> Path:
    """<outdir>/step_NNNNNN, the reference's per-export directory."""
    return Path(outdir) / f"step_{int(index):06d}"


class HistoryWriter:
    """Writes history frames of ResidentRun / EngineRun members in the
    background.  fields: names from cuda.HISTORY_FIELDS; buffers: pinned images
    in flight at once."""

    def __init__(self, ctx: cuda.Context, fields=cuda.HISTORY_FIELDS, buffers: int = 3):
        self.ctx = ctx
        self.mask = cuda.history_mask(fields)
        self.count = bin(self.mask).count("1")
        self._limit = max(1, int(buffers))
        self._made = 0
        self._free: queue.Queue = queue.Queue()
        self._work: queue.Queue = queue.Queue()
        self.errors: list = []
        self.frames = 0
        self.bytes_written = 0
        self._thread = threading.Thread(target=self._drain, name="nimbus-history", daemon=True)
        self._thread.start()

    def _image(self, floats: int) -> np.ndarray:
        if self._free.empty() and self._made < self._limit:
            self._made += 1
            img = torch.empty(floats, dtype=torch.float32).pin_memory().numpy()
        else:
            img = self._free.get()
        if img.size < floats:
            img = torch.empty(floats, dtype=torch.float32).pin_memory().numpy()
        return img

    def _submit(self, img, shape, stream_handle: int, directory: Path):
        event = torch.cuda.Event()
        event.record(torch.cuda.ExternalStream(stream_handle))
        self._work.put((img, tuple(shape), event, Path(directory)))

    def frame(self, run, index: int, outdir) -> Path:
        """Enqueue a frame of a ResidentRun (after the steps already enqueued on
        its stream) into <outdir>/step_NNNNNN; returns that directory."""
        shape = run.case.shape
        img = self._image(self.count * run.cells)
        args = cuda.history_args(run.fields, self.mask, img, shape, stream=run.stream)
        self.ctx.check(self.ctx.history_snapshot(args))
        directory = frame_dir(outdir, index)
        self._submit(img, shape, run.stream, directory)
        return directory

    def frame_member(self, engine_run, member_id: int, index: int, outdir) -> Path:
        """Enqueue a frame of one engine member (after the engine's enqueued steps)."""
        engine = engine_run.engine
        shape = engine.shapes[member_id]
        img = self._image(self.count * shape[0] * shape[1] * shape[2])
        engine.history_async(member_id, self.mask, img)
        directory = frame_dir(outdir, index)
        self._submit(img, shape, engine.stream, directory)
        return directory

    def _drain(self):
        while True:
            item = self._work.get()
            if item is None:
                self._work.task_done()
                return
            img, shape, event, directory = item
            try:
                event.synchronize()
                shutil.rmtree(directory, ignore_errors=True)
                directory.mkdir(parents=True, exist_ok=True)
                rc = cuda.history_write(img, self.mask, shape, directory, self.ctx.lib)
                if rc != cuda.NIMBUS_OK:
                    self.errors.append(f"{directory}: {cuda.STATUS_NAMES.get(rc, rc)}")
                else:
                    self.frames += 1
                    self.bytes_written += self.count * shape[0] * shape[1] * shape[2] * 4
            except Exception as exc:  # reported by flush()
                self.errors.append(f"{directory}: {exc}")
            finally:
                self._free.put(img)
                self._work.task_done()

    def flush(self):
        """Wait until every enqueued frame is on disk; raise on any failure."""
        self._work.join()
        if self.errors:
            raise RuntimeError("history write failed: " + "; ".join(self.errors))

    def close(self):
        self.flush()
        self._work.put(None)
        self._thread.join()
