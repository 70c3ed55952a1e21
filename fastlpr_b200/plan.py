"""Many LPR fits in one captured CUDA graph.

    plan = LprPlan([(x1, y1, h1, opts1), (x2, y2, h2, opts2), ...])
    regs = plan.run()                  # the responses given above
    regs = plan.run([y1b, y2b, ...])   # new responses on the same designs

No reference counterpart: the reference fits one data set per call
(api.py:167-832).  Every problem is validated like ``cv_fastlpr`` and gives
the same result (full GCV sweep).  What depends on x only -- point
statistics, grid geometry, kernel spectra, the bandwidth filter, probes --
is formed when the plan is built; everything that reads y -- spread and
transform of every channel, deposits, convolutions, solves, GCV/DoF
reductions, the 1-SE choice, the fitted values at the chosen bandwidth and
the copies of every output into pinned host buffers -- is captured once into
a CUDA graph and replayed by ``run``.  The problems are spread over several
streams inside the graph (largest first, each to the least loaded stream),
so small and large data sets of uneven size run concurrently.  A plan of
many full-sweep problems is captured as a few graphs over consecutive
parts of that order (about 1/8, 1/8, 1/4 and 1/2 of the response bytes),
each replayed on its own stream as soon as its responses are staged: the
host stages the later parts while the device fits the earlier ones.  A run
is one replay of each graph and one synchronisation for all problems.

``cv_fastlpr_many`` runs a list of problems once (eagerly, on the same
streams, no capture).
"""
from __future__ import annotations

import collections
import os
import time
from concurrent.futures import ThreadPoolExecutor
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib, api
from .structures import RegressionOutput


class _Problem:
    pass


class _Segment:
    """One captured graph: the problems it fits (issue order), their
    captured outputs, its NaN/Inf flag and the stream it replays on."""

    def __init__(self, idx, graph, outs, finite, stream):
        self.idx = idx
        self.graph = graph
        self.outs = outs
        self.finite = finite
        self.stream = stream


def _cost(p) -> float:
    """Relative device time of one fit: per-point spreading plus the
    per-bandwidth convolutions on the padded grid."""
    L = float(np.prod(p.geom.L.astype(float)))
    nprod = (len(api._element_powers(p.d, p.su.order)) + (p.su.dy + 10) *
             (1 if p.su.order == 0 else len(api._design_powers(p.d, p.su.order))))
    return p.su.n * (p.su.dy + 11) * (3 ** p.d) + len(p.filt[2]) * nprod * L


def estimated_cost(x, y, h, options) -> float:
    """Relative device time of one problem from its sizes alone (points,
    dimension, order, response channels, bandwidths, padded grid), for
    splitting a set of problems between GPUs before any work is done."""
    x = np.asarray(x)
    n = x.shape[0]
    d = 1 if x.ndim == 1 else x.shape[1]
    opts = dict(options or {})
    order = int(opts.get("order", 0))
    dy = (1 if np.asarray(y).ndim == 1 else np.asarray(y).shape[1]) * \
        (2 if np.iscomplexobj(y) else 1)
    G = api._grid_shape(opts, n, d)
    L = 2.0 ** np.ceil(np.log2(2 * G - 1))
    H = np.atleast_2d(np.asarray(h)).shape[0]
    nprod = (len(api._element_powers(d, order)) + (dy + 10) *
             (1 if order == 0 else len(api._design_powers(d, order))))
    return float(n * (dy + 11) * (3 ** d) + H * nprod * np.prod(L) * (2.0 if order == 2 else 1.0))


def partition_by_cost(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Indices split into `parts` groups of similar total cost (largest
    first, each to the least loaded group)."""
    groups: List[List[int]] = [[] for _ in range(max(1, parts))]
    load = [0.0] * len(groups)
    for i in sorted(range(len(costs)), key=lambda i: -costs[i]):
        k = int(np.argmin(load))
        groups[k].append(i)
        load[k] += costs[i]
    return [sorted(g) for g in groups]


class LprPlan:
    """A set of LPR fits captured as one CUDA graph (see the module docstring).

    problems: sequence of (x, y, h, options) exactly as for cv_fastlpr
    (h explicit).  Problems with bandwidth_search='learned' take the
    learned search: binned sums, features, the network (one batch for all
    of them) and the window choice run inside the graph, and each evaluates
    its five-bandwidth window there; acceptance is checked after the replay
    and the rare walks or full-sweep fallbacks run eagerly.
    streams: concurrent streams inside the graph (default: up to 8).
    graph: capture a CUDA graph (True) or issue eagerly on every run.
    autotune: pick the number of streams and the spread work-item size by
    timing graph replays of this plan (cached per workload signature, see
    fastlpr_b200.autotune); the spread setting stays applied afterwards.
    """

    def __init__(self, problems: Sequence, device=None, streams: Optional[int] = None,
                 graph: bool = True, autotune: bool = False):
        if len(problems) == 0:
            raise ValueError("LprPlan needs at least one problem")
        self.device = torch.device(device) if device is not None else api._device({})
        self.probs: List[_Problem] = []
        with torch.cuda.device(self.device):
            ctx = api._Ctx(self.device)
            self._ctx = ctx
            setups = []
            for (x, y, h, options) in problems:
                opts = dict(options or {})
                if str(opts.get("bandwidth_search", "full")) not in ("full", "learned"):
                    raise ValueError(f"bandwidth_search must be 'full' or 'learned', got "
                                     f"{opts.get('bandwidth_search')!r}")
                opts["device"] = str(self.device)
                if h is None:
                    raise ValueError("LprPlan needs explicit bandwidths for every problem")
                setups.append(api._lpr_setup(x, y, h, opts))
            # probes: one cached matrix per (R, seed) covering the largest n
            nmax = max(s.n for s in setups)
            for su in setups:
                if bool(su.opts.get("calc_dof", True)) and su.opts.get("random_matrix") is None:
                    api._probes(ctx, nmax, int(su.opts.get("num_dof_sample", 10)),
                                su.opts.get("dof_seed", 42), None)
            for su in setups:
                self.probs.append(self._build(ctx, su))
            self._setup_learned()
            self._pool = None
            self._finite = None
            self._write_y([p.su.y_arr for p in self.probs], range(len(self.probs)))
            for p in self.probs:
                self._check_finite(bool(np.all(np.isfinite(p.staging.numpy()))))
            # downloads of each problem's outputs, issued behind its last
            # kernel (an event recorded in the graph) so they overlap the
            # rest of the replay
            self._copy = torch.cuda.Stream(self.device)
            # whether the responses on the device passed their NaN/Inf check
            # (a rejected run leaves them there; a replay without new
            # responses would fit them)
            self._y_ok = True
            self.segs = None
            self._graph_downloads = False
            self.tuning = None
            if autotune and graph:
                self.tuning = self._autotune()
                streams = self.tuning["best"]["streams"]
            self._set_streams(streams if streams is not None else min(8, len(self.probs)))
            if graph:
                self._capture()

    def _workers(self) -> ThreadPoolExecutor:
        """The host threads that stage responses and build results (started
        again after close)."""
        if self._pool is None:
            self._pool = ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1)))
        return self._pool

    def close(self) -> None:
        """Stop the staging threads (also done when the plan is collected)."""
        pool, self._pool = getattr(self, "_pool", None), None
        if pool is not None:
            pool.shutdown(wait=False)

    def __del__(self):
        self.close()

    def _set_streams(self, nstreams: int) -> None:
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max(1, int(nstreams)))]
        # largest first, each to the least loaded stream
        order = sorted(range(len(self.probs)), key=lambda i: -_cost(self.probs[i]))
        load = [0.0] * len(self.streams)
        self.assign = {}
        for i in order:
            k = int(np.argmin(load))
            self.assign[i] = k
            load[k] += _cost(self.probs[i])
        self.order = order

    def _segment_order(self) -> List[List[int]]:
        """The issue order cut into consecutive parts of about 1/8, 1/8, 1/4
        and 1/2 of the staged response bytes (one part for fewer than eight
        problems or when the learned proposal chain joins all problems)."""
        if self.prop is not None or len(self.order) < 8:
            return [list(self.order)]
        sizes = [self.probs[i].staging.numel() for i in self.order]
        total = float(sum(sizes))
        bounds = (total / 8, total / 4, total / 2)
        segs = [[] for _ in range(len(bounds) + 1)]
        acc = 0.0
        for i, sz in zip(self.order, sizes):
            segs[sum(acc >= b for b in bounds)].append(i)
            acc += sz
        return [sg for sg in segs if sg]

    def _capture(self) -> None:
        # eager pass: cuFFT plans, kernel attributes, output buffers
        outs = self._issue(self.order)
        torch.cuda.synchronize(self.device)
        if self.prop is None:
            # full sweeps: every output also gets a pinned buffer of the plan,
            # so each problem's downloads are captured on its own stream
            # right behind its last kernel
            for i, p in enumerate(self.probs):
                for k, t in outs[i][2].items():
                    if isinstance(t, torch.Tensor) and t.is_cuda:
                        p.bufs[k] = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            self._graph_downloads = True
        del outs
        # one graph per part, each with its own memory pool (the parts'
        # replays overlap on the device)
        self.segs = []
        for idx in self._segment_order():
            graph = torch.cuda.CUDAGraph()
            cap = torch.cuda.Stream(self.device)
            cap.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.graph(graph, stream=cap):
                outs = self._issue(idx)
            self.segs.append(_Segment(idx, graph, outs, self._finite,
                                      torch.cuda.Stream(self.device)))
        torch.cuda.synchronize(self.device)

    def replay(self) -> None:
        """Replay every captured graph on the staged responses (each on its
        stream, joined back into the current stream)."""
        main = torch.cuda.current_stream(self.device)
        for sg in self.segs:
            sg.stream.wait_stream(main)
            with torch.cuda.stream(sg.stream):
                sg.graph.replay()
        for sg in self.segs:
            main.wait_stream(sg.stream)

    def _autotune(self) -> dict:
        """Streams x spread work-item size, timed as graph replays."""
        from . import autotune as at
        sig = sorted((p.d, tuple(int(v) for v in p.geom.L), p.su.order, p.su.dy,
                      p.su.y_is_complex, int(np.round(np.log2(p.su.n))), len(p.filt[2]))
                     for p in self.probs)
        key = "plan|" + at.device_key(self.device) + "|" + str(hash(tuple(sig)) & 0xFFFFFFFF)
        saved = at.get_params()
        cands = [{"streams": s, "spread_item_points": a}
                 for s in (2, 4, 8, 16) if s <= max(2, len(self.probs))
                 for a in at.ITEM_POINTS]

        def measure(c):
            at.set_params({"spread_item_points": c["spread_item_points"]})
            self._set_streams(c["streams"])
            self._capture()
            ms = at.time_ms(self.replay, device=self.device)
            self.segs = None
            return ms

        try:
            rec = at.tune(key, cands, measure)
        finally:
            at.set_params(saved)
        at.set_params({"spread_item_points": rec["best"]["spread_item_points"]})
        return rec

    # -- construction -------------------------------------------------------
    def _setup_learned(self) -> None:
        """Problems with bandwidth_search='learned' that the proposal network
        serves (one real response, d <= 2, Gaussian kernel, DoF on, an
        increasing isotropic bandwidth list none of which the grid filter
        removes) share one device proposal chain (learned.DeviceProposal);
        the others run the full sweep."""
        from . import learned as _learned
        self.prop = None
        metas, lhs = [], []
        for p in self.probs:
            su = p.su
            p.lidx = None
            p.search = None
            if str(su.opts.get("bandwidth_search", "full")) != "learned":
                continue
            # what a single learned fit records when the network does not
            # serve the problem
            p.search = {"mode": "learned", "accepted": False, "fallback": "full sweep"}
            lh = _learned.isotropic_log_h(su.bandwidths)
            ok = (lh is not None and bool(su.opts.get("calc_dof", True)) and su.dy == 1
                  and not su.y_is_complex and su.d <= 2 and api._kernel_id(su.opts) == 0
                  and len(p.filt[2]) == su.bandwidths.shape[0])
            if not ok:
                continue
            p.lidx = len(metas)
            metas.append((su.d, su.order, su.n))
            lhs.append(lh)
            p.dstats = torch.from_numpy(np.ascontiguousarray(p.stats[:2].ravel())).to(self.device)
        if metas:
            model = _learned.default_model(self.device)
            self.prop = _learned.DeviceProposal(model, metas, lhs, self.device)
            self.lo_h = torch.empty(len(metas), dtype=torch.int32, pin_memory=True)
            self.t_h = torch.empty(len(metas), dtype=torch.float64, pin_memory=True)

    def _build(self, ctx, su) -> _Problem:
        p = _Problem()
        p.su = su
        p.d = su.d
        x = su.x_arr
        if not np.all(np.isfinite(x)):
            raise ValueError("Input x contains NaN or Inf values")
        p.dx = ctx.upload(x)
        p.stats = api._point_stats(ctx, p.dx, su.n, su.d)
        G = api._grid_shape(su.opts, su.n, su.d)
        p.geom = api._make_geom(p.stats, su.n, su.d, G, int(su.opts["accuracy"]),
                                bool(su.opts.get("flag_power2", True)))
        p.filt = api._filter_bandwidths(ctx, p.geom, su.bandwidths, 2 * su.order + 1,
                                        api._kernel_id(su.opts))
        bw_k = p.filt[1][p.filt[2]]
        hs = torch.from_numpy(np.ascontiguousarray(np.sum(bw_k, axis=1)))
        p.hsum = hs.to(self.device)
        p.bufs = None
        p.probes = None
        if bool(su.opts.get("calc_dof", True)):
            p.probes = api._probes(ctx, su.n, int(su.opts.get("num_dof_sample", 10)),
                                   su.opts.get("dof_seed", 42), su.opts.get("random_matrix"))
        methods = api._check_interp_methods(su.opts, su.d, su.n)
        if "cubic" in methods.values():
            from . import spline
            spline.tables(api._raw_axes(p.geom, su.opts), ctx.device)
        nch = su.dy * (2 if su.y_is_complex else 1)
        p.ycols = [torch.zeros(su.n, dtype=torch.float64, device=self.device) for _ in range(nch)]
        p.staging = torch.empty((nch, su.n), dtype=torch.float64, pin_memory=True)
        return p

    def _check_y(self, ys) -> list:
        """The responses as (n, dy) arrays, checked against the plan."""
        if len(ys) != len(self.probs):
            raise ValueError(f"expected {len(self.probs)} responses, got {len(ys)}")
        arrs = []
        for p, y in zip(self.probs, ys):
            y_arr = np.asarray(y)
            if y_arr.ndim == 1:
                y_arr = y_arr[:, None]
            elif y_arr.ndim == 2 and y_arr.shape[0] == 1 and y_arr.shape[1] > 1:
                y_arr = y_arr.T
            if y_arr.shape != p.su.y_arr.shape:
                raise ValueError(f"response shape {y_arr.shape} differs from the planned "
                                 f"{p.su.y_arr.shape}")
            if bool(np.iscomplexobj(y_arr)) != p.su.y_is_complex:
                raise ValueError("a response changed between real and complex")
            arrs.append(y_arr)
        return arrs

    def _write_y(self, arrs, idx) -> None:
        """Copy the responses of problems `idx` into their pinned staging
        rows (a few host threads: numpy's copies release the GIL).  The
        upload to the device and the NaN/Inf check are part of the issued
        work (_upload_y), so in a graph they overlap the other problems'
        kernels."""

        def stage(i):
            p, y_arr = self.probs[i], arrs[i]
            st = p.staging.numpy()
            for c in range(p.su.dy):
                if p.su.y_is_complex:
                    st[2 * c] = y_arr[:, c].real
                    st[2 * c + 1] = y_arr[:, c].imag
                else:
                    st[c] = y_arr[:, c]

        list(self._workers().map(stage, idx))

    @staticmethod
    def _upload_y(p) -> torch.Tensor:
        """On the current stream: the staged responses of problem p to its
        device columns, and whether all of them are finite (device flag)."""
        for c, col in enumerate(p.ycols):
            col.copy_(p.staging[c], non_blocking=True)
        return torch.isfinite(torch.stack(p.ycols)).all()

    @staticmethod
    def _check_finite(flag) -> None:
        if flag is not None and not bool(flag):
            raise ValueError("Response y contains NaN or Inf values")

    def _issue(self, idx) -> dict:
        """Enqueue the y-dependent stages of problems `idx` (issue order) on
        their streams, up to their outputs in the pinned buffers; returns
        {problem: (state, results, pending outputs)}.  Problems with the learned
        search stop after their binned sums; the proposal chain then runs
        once for all of them on the main stream, and each evaluates the
        window it chose (kernel factors gathered on the device) up to its
        outputs."""
        main = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(main)
        outs = {}
        states = {}
        flags = []
        for i in idx:
            p = self.probs[i]
            su = p.su
            if getattr(p, "done", None) is None:
                p.done = torch.cuda.Event(external=True)
            with torch.cuda.stream(self.streams[self.assign[i]]):
                flags.append(self._upload_y(p))
                ctx = api._Ctx(self.device)
                ev = api._PhaseEvents(None)
                st = api._prepare_lpr(ctx, None, None, su.dy, su.opts, su.order, su.prec,
                                      su.variance, su.y_is_complex, (p.dx, list(p.ycols)),
                                      ev, stats=p.stats, probes=p.probes,
                                      bandwidths=su.bandwidths)
                if p.lidx is not None:
                    _lib.check(ctx.lib.flpr_bin_moments(
                        su.d, su.n, p.dx.data_ptr(), st.ycols[0].data_ptr(), p.dstats.data_ptr(),
                        self.prop.bins[p.lidx].data_ptr(), ctx.stream), "flpr_bin_moments")
                    states[i] = st
                    continue
                r = api._evaluate_device(ctx, st, p.filt, ev)
                if p.bufs is None:
                    p.bufs = api._output_bufs(st, r["H"])
                pend = api._finalize_enqueue(ctx, st, r, ev, device_select=True, bufs=p.bufs,
                                             hsum_dev=p.hsum)
                p.done.record()
                outs[i] = (st, r, pend)
        if states:
            from . import learned as _learned
            for s in self.streams:
                main.wait_stream(s)
            self.prop.enqueue(main.cuda_stream)
            self.lo_h.copy_(self.prop.lo, non_blocking=True)
            self.t_h.copy_(self.prop.t, non_blocking=True)
            for s in self.streams:
                s.wait_stream(main)
            for i in idx:
                if i not in states:
                    continue
                p, st = self.probs[i], states[i]
                with torch.cuda.stream(self.streams[self.assign[i]]):
                    ctx = api._Ctx(self.device)
                    ev = api._PhaseEvents(None)
                    filt_w, hsum, _ = api._window_filter(
                        ctx, st, p.filt, self.prop.lo[p.lidx:p.lidx + 1], _learned.REFINE)
                    r = api._evaluate_device(ctx, st, filt_w, ev)
                    if p.bufs is None:
                        p.bufs = api._output_bufs(st, r["H"])
                    pend = api._finalize_enqueue(ctx, st, r, ev, device_select=True,
                                                 bufs=p.bufs, hsum_dev=hsum)
                    p.done.record()
                    outs[i] = (st, r, pend)
        for s in self.streams:
            main.wait_stream(s)
        self._finite = torch.stack(flags).all().reshape(1)
        return outs

    # -- execution ----------------------------------------------------------
    def run(self, ys: Optional[Sequence] = None,
            timings: Optional[dict] = None) -> List[RegressionOutput]:
        """Fit every problem (with new responses `ys` if given).  timings
        (optional dict): accumulates host wall seconds of the stages
        'stage' (responses into the pinned staging rows and the graphs
        launched), 'enqueue' (downloads issued, results built as they
        arrive), 'wait' (device done) and 'results' (the remaining
        results)."""
        clock = [time.perf_counter()]

        def mark(name):
            if timings is not None:
                now = time.perf_counter()
                timings[name] = timings.get(name, 0.0) + now - clock[0]
                clock[0] = now

        with torch.cuda.device(self.device):
            if ys is None and not self._y_ok:
                raise ValueError("Response y contains NaN or Inf values (the last responses "
                                 "given to run were rejected; pass new responses)")
            arrs = self._check_y(ys) if ys is not None else None
            main = torch.cuda.current_stream(self.device)
            if self.segs is not None:
                # each part's graph starts as soon as its responses are staged
                outs = {}
                for sg in self.segs:
                    if arrs is not None:
                        self._write_y(arrs, sg.idx)
                    sg.stream.wait_stream(main)
                    with torch.cuda.stream(sg.stream):
                        sg.graph.replay()
                    outs.update(sg.outs)
                for sg in self.segs:
                    main.wait_stream(sg.stream)
                flag = (self.segs[0].finite if len(self.segs) == 1 else
                        torch.cat([sg.finite for sg in self.segs]).all().reshape(1))
            else:
                if arrs is not None:
                    self._write_y(arrs, range(len(self.probs)))
                outs = self._issue(self.order)
                flag = self._finite
            mark("stage")
            finite = api._to_host(flag)
            if self._graph_downloads:
                return self._collect(outs, finite, main, mark)
            # each problem's outputs go into fresh pinned memory (no host
            # copies; the results stay valid after later runs) on the copy
            # stream, as soon as that problem's last kernel is done (in issue
            # order, which is about the order the problems finish).  The
            # full-sweep results are built while the device still works on
            # later problems; the NaN/Inf check of the responses comes after
            # all of them (results of rejected responses are dropped, and a
            # build that fails before the check is repeated after it).
            pends, done = {}, {}
            res = [None] * len(self.probs)
            ready, deferred = collections.deque(), []
            ev = api._PhaseEvents(None)

            def build(i):
                p = self.probs[i]
                st, r, _ = outs[i]
                return api._finalize_build(self._ctx, st, r, pends[i], ev,
                                           dict(p.search) if p.search else None)

            def drain(block):
                while ready and (block or done[ready[0]].query()):
                    i = ready.popleft()
                    done[i].synchronize()
                    try:
                        res[i] = build(i)
                    except Exception:  # noqa: BLE001 - repeated after the check
                        deferred.append(i)

            with torch.cuda.stream(self._copy):
                for i in self.order:
                    p = self.probs[i]
                    st, r, pend = outs[i]
                    self._copy.wait_event(p.done)
                    pends[i] = {k: (api._to_host(v) if isinstance(v, torch.Tensor)
                                    and v.is_cuda else v) for k, v in pend.items()}
                    if p.lidx is None:
                        done[i] = torch.cuda.Event()
                        done[i].record(self._copy)
                        ready.append(i)
                    drain(False)
            mark("enqueue")
            main.synchronize()
            self._copy.synchronize()
            mark("wait")
            drain(True)
            self._y_ok = bool(finite[0])
            self._check_finite(finite[0])
            for i in deferred:
                res[i] = build(i)
            for i, p in enumerate(self.probs):
                if p.lidx is not None:
                    st, r, _ = outs[i]
                    res[i] = self._finish_learned(p, st, r, pends[i], ev)
            mark("results")
            return res

    def _collect(self, outs, finite, main, mark) -> List[RegressionOutput]:
        """Results of a replay whose downloads are in the graphs: as each
        problem's event fires (issue order) a worker thread builds its
        result, copying the outputs out of the plan's pinned buffers (the
        results stay valid after later runs).  The NaN/Inf check of the
        responses comes after all of them; a build that failed before it is
        repeated after it."""
        ev = api._PhaseEvents(None)

        def build(i):
            p = self.probs[i]
            st, r, pend = outs[i]
            return api._finalize_build(self._ctx, st, r, pend, ev,
                                       dict(p.search) if p.search else None, copy=True)

        def attempt(i):
            try:
                return build(i), None
            except Exception as exc:  # noqa: BLE001 - repeated after the check
                return None, exc

        futs = {}
        for i in self.order:
            self.probs[i].done.synchronize()
            futs[i] = self._workers().submit(attempt, i)
        mark("enqueue")
        main.synchronize()
        mark("wait")
        res = [None] * len(self.probs)
        failed = []
        for i, f in futs.items():
            res[i], exc = f.result()
            if exc is not None:
                failed.append(i)
        self._y_ok = bool(finite[0])
        self._check_finite(finite[0])
        for i in failed:
            res[i] = build(i)
        mark("results")
        return res

    def _finish_learned(self, p, st, r, pend, ev) -> RegressionOutput:
        """Acceptance of a learned problem's window after the replay; the
        rare walks and full-sweep fallbacks run eagerly on its prepared state
        (valid until the next replay)."""
        ctx = self._ctx
        bw = p.su.bandwidths
        # FP64 spectra formed eagerly after an earlier replay hold that
        # replay's responses: form them again from this replay's grid
        st.spec64 = None
        found = api._learned_finish(ctx, st, bw, dict(r), pend, int(self.lo_h[p.lidx]),
                                    float(self.t_h[p.lidx]), ev)
        if found is None:
            return api._full_sweep(ctx, st, bw, ev, {"mode": "learned", "accepted": False,
                                                      "fallback": "full sweep"}, filt=p.filt)
        r2, record, pend2 = found
        if pend2 is not None:
            return api._finalize_build(ctx, st, r2, pend2, ev, record)
        return api._finalize_lpr(ctx, st, r2, ev, record)


def cv_fastlpr_many(problems: Sequence, device=None,
                    streams: Optional[int] = None) -> List[RegressionOutput]:
    """cv_fastlpr for every (x, y, h, options) of `problems`, issued on
    concurrent streams with one synchronisation for the reductions and one
    for the outputs.  Same results as separate cv_fastlpr calls."""
    return LprPlan(problems, device=device, streams=streams, graph=False).run()
