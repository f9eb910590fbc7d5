"""Batched shots over the vi_batch C ABI: many shots of different grids and
step counts advance together, one launch per time step for all of them,
the whole run one CUDA graph.  The reference solves one problem per call
(sciml_solver/ViscoelasticProblem.jl:273-309); this is its time step run
for a whole gather of shots at once."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._abi import (ViConfig, ViFields, ViMedium, VI_BATCH_NO_GRAPH, VI_BATCH_RETUNE, check, lib)
from .solver import MEDIUM_NAMES, StepPlan, config_from_workload, _stream_handle


class ShotBatch:
    """Device-resident batch of shots built from media.Workload objects."""

    def __init__(self, workloads, precision: str = "f32", device=None):
        self.workloads = list(workloads)
        n = len(self.workloads)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.dtype = torch.float64 if precision == "f64" else torch.float32
        cfgs = (ViConfig * n)(*[config_from_workload(w, precision) for w in self.workloads])
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(lib().vi_batch_create(cfgs, n, C.byref(self._h)))
        self.media, self.states, self.wavelets, self.traces = [], [], [], []
        self._keep = []
        for i, w in enumerate(self.workloads):
            kw = dict(device=self.device, dtype=self.dtype)
            med = {k: torch.as_tensor(np.ascontiguousarray(v), **kw) for k, v in w.medium.items()}
            st = {"v": torch.zeros(2, w.nz, w.nx, **kw), "s": torch.zeros(3, w.nz, w.nx, **kw),
                  "m": torch.zeros(3, max(w.nsls, 1), w.nz, w.nx, **kw)}
            wav = torch.as_tensor(w.wavelets[:, :w.nt], **kw).contiguous()
            tr = torch.zeros(2, len(w.receivers), w.nt, **kw)
            self.media.append(med)
            self.states.append(st)
            self.wavelets.append(wav)
            self.traces.append(tr)
            m = ViMedium()
            for k in MEDIUM_NAMES:
                if k in med:
                    setattr(m, k, med[k].data_ptr())
            f = StepPlan.fields_struct(st["v"][0], st["v"][1], st["s"][0], st["s"][1], st["s"][2],
                                       st["m"] if w.nsls else None)
            shot, keep = StepPlan._shot(None, w.sources, wav, w.receivers, tr)
            self._keep.append((m, f, shot, keep))
            check(lib().vi_batch_set_shot(self._h, i, C.byref(m), C.byref(f), C.byref(shot), w.nt))

    def __len__(self):
        return len(self.workloads)

    def run(self, graph: bool = True, retune: bool = False, stream=None):
        flags = (0 if graph else VI_BATCH_NO_GRAPH) | (VI_BATCH_RETUNE if retune else 0)
        check(lib().vi_batch_run(self._h, flags, _stream_handle(stream)))

    def status(self, stream=None) -> str:
        form = C.c_int32()
        check(lib().vi_batch_status(self._h, _stream_handle(stream), C.byref(form)))
        return {4: "streams", 3: "per-shot", 2: "split", 1: "two-stage", 0: "one-stage", -1: "untuned"}[form.value]

    def reset(self):
        """Zeroes every shot's wavefields and traces (rest state)."""
        for st, tr in zip(self.states, self.traces):
            for t in st.values():
                t.zero_()
            tr.zero_()

    def result(self, i):
        """(traces [2, nrec, nt], state) of shot i as float64 numpy arrays."""
        st = {k: v.double().cpu().numpy() for k, v in self.states[i].items()}
        st["m"] = st["m"].reshape(-1, self.workloads[i].nz, self.workloads[i].nx)
        return self.traces[i].double().cpu().numpy(), st

    def point_steps(self) -> int:
        return sum(w.nx * w.nz * w.nt for w in self.workloads)

    def close(self):
        if self._h:
            lib().vi_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
