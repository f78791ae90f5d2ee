"""Systems workloads over the evaluator: the batched uneven mix and the serving loop.

Batched uneven workload: many ciphertexts of different ring degree and live
limb count with a mix of HMult + relinearise + rescale, rotations and
additions.  The grouped schedule runs one context (stream) per ring degree,
batches every HMult of a degree into grouped launches (aoa_hmult_batch groups
by limb count) and every rotation of the degree into one batched call
(aoa_rotate_batch_steps, grouped by limb count, a step and key per op), and is captured
once per context into a CUDA graph that is replayed; the plain schedule
issues the reference's per-call operation sequence one op at a time.

Serving loop: requests (a plaintext-weight multiply with rescale, a
rotate-and-sum over the slots, a rescale) arrive as a Poisson process;
requests are admitted while a slot (a context of the request's ring degree)
and the HBM budget allow, run asynchronously next to the requests already on
the device, and complete in any order.  Keys stay resident and count against
the budget first (they dominate it: 15 Galois keys of 2 x 61 limbs at 2^16
are 0.94 GB); a request's three ciphertexts count while it is in flight.
Latency is arrival to completion on the host clock; each run records how
many requests were admitted and how many had to wait for a slot or for
budget.
"""
import time

import numpy as np

from . import (AOA_COEF, AOA_NTT, Ciphertext, Context, Engine, Graph, SwitchKey, ckks_add, ckks_encode,
               ckks_mul_batch, ckks_mul_plain, ckks_mul_pt, ckks_rescale, ckks_rotate_batch, ckks_rotate_batch_steps,
               ckks_rotate_plain, ckks_sumslots, params)


def _rand_residues(rng, primes, n):
    return np.array([rng.integers(0, q, n, dtype=np.uint64) for q in primes], dtype=np.uint64)


def hbm_bytes(op, m, kl, n):
    """Algorithmic HBM bytes of one op with m live limbs (fused lower bound)."""
    if op == "mul":
        return (4 * m + 2 * (m + kl) + 2 * (m - 1)) * n * 8
    if op == "rot":
        return (2 * m + 2 * (m + kl) + 2 * m) * n * 8
    return 6 * m * n * 8



# 60-bit primes q = 1 mod 2^32 (q = 1 mod 2N for every degree used): their
# limb transforms take the shorter Shoup remainder
PRIME_MODULUS = 1 << 32


class UnevenBatch:
    """The batched uneven workload: n_ops ops over ring degrees 2^log_ns, live
    limbs uniform in [min_limbs, k], op mix mul / rot / add."""

    def __init__(self, n_ops=512, seed=4, log_ns=(14, 15, 16), k=30, kl=31, min_limbs=4, mix=(0.5, 0.3, 0.2),
                 inputs_per_n=4, scale_bits=50, autotune=False):
        rng = np.random.default_rng(seed)
        self.k, self.kl = k, kl
        primes = params.ntt_primes(60, PRIME_MODULUS, k + kl)
        self.engines, self.ctx, self.evk, self.rtk, self.inputs = {}, {}, {}, {}, {}
        for ln in log_ns:
            E = Engine(ln, primes[:k], primes[k:], scale_bits=scale_bits)
            if autotune:
                E.autotune()                  # transform launch shapes picked per ring degree
            ctx = Context(E)
            N = 1 << ln
            self.engines[ln], self.ctx[ln] = E, ctx
            self.evk[ln] = SwitchKey(ctx, _rand_residues(rng, primes, N), _rand_residues(rng, primes, N))
            # a distinct rotation key for every step 2^j the mix can draw (the reference's
            # ckks_new_rtk_left makes one per power of two, ckkskeys.cpp:146-181): the key
            # traffic of distinct keys is paid as in a real mix
            self.rtk[ln] = {1 << j: SwitchKey(ctx, _rand_residues(rng, primes, N), _rand_residues(rng, primes, N))
                            for j in range(ln - 1)}
            self.inputs[ln] = [Ciphertext.from_residues(ctx, _rand_residues(rng, primes[:k], N),
                                                        _rand_residues(rng, primes[:k], N), slots=N // 2,
                                                        scale=1 << scale_bits, domain=AOA_NTT)
                               for _ in range(inputs_per_n)]
        self.scale = 1 << scale_bits
        self.ops = []
        kinds = rng.choice(["mul", "rot", "add"], size=n_ops, p=list(mix))
        for z in range(n_ops):
            ln = int(rng.choice(log_ns))
            m = int(rng.integers(min_limbs, k + 1))
            step = 1 << int(rng.integers(0, ln - 1))
            a, b = rng.integers(0, inputs_per_n, 2)
            self.ops.append({"kind": str(kinds[z]), "log_n": ln, "m": m, "step": step, "a": int(a), "b": int(b)})
        self.outs = [Ciphertext(self.ctx[op["log_n"]]) for op in self.ops]
        # every op owns its operands (device copies of the degree's templates)
        self.args = []
        for op in self.ops:
            ins = self.inputs[op["log_n"]]
            n_in = 1 if op["kind"] == "rot" else 2
            self.args.append([ins[op["a"]].copy()] + ([ins[op["b"]].copy()] if n_in == 2 else []))
        self.sync()
        self.bytes = sum(hbm_bytes(op["kind"], op["m"], kl, 1 << op["log_n"]) for op in self.ops)
        self.graphs = None

    def _args(self, z, domain=AOA_NTT):
        op = self.ops[z]
        for ct in self.args[z]:
            ct.set(op["m"] - 1, ct.slots, self.scale, domain)
        return self.args[z]

    def run_grouped(self, ln):
        """Every op of degree 2^ln on its context: the HMults in grouped batched
        launches (grouped by limb count inside the call), the rotations in one
        batched call (grouped by limb count inside the call, each op with its
        own step and key), then the additions."""
        ctx = self.ctx[ln]
        muls = [z for z, op in enumerate(self.ops) if op["log_n"] == ln and op["kind"] == "mul"]
        if muls:
            pairs = [self._args(z) for z in muls]
            ckks_mul_batch(ctx, [self.outs[z] for z in muls], [p[0] for p in pairs], [p[1] for p in pairs],
                           self.evk[ln])
        rots = [z for z, op in enumerate(self.ops) if op["log_n"] == ln and op["kind"] == "rot"]
        if rots:                    # one call: grouped by limb count, a step and key per op
            ckks_rotate_batch_steps(ctx, [self.outs[z] for z in rots], [self._args(z)[0] for z in rots],
                                    [self.ops[z]["step"] for z in rots],
                                    [self.rtk[ln][self.ops[z]["step"]] for z in rots])
        for z, op in enumerate(self.ops):
            if op["log_n"] == ln and op["kind"] == "add":
                args = self._args(z)
                ckks_add(ctx, self.outs[z], args[0], args[1])

    def run_plain(self):
        """The reference's per-call sequence, one op at a time in input order
        (HMult and rotations through the reference-structured paths)."""
        for z, op in enumerate(self.ops):
            ln = op["log_n"]
            ctx = self.ctx[ln]
            args = self._args(z)
            if op["kind"] == "mul":
                ckks_mul_plain(ctx, self.outs[z], args[0], args[1], self.evk[ln])
            elif op["kind"] == "rot":
                ckks_rotate_plain(ctx, self.outs[z], args[0], op["step"], self.rtk[ln][op["step"]])
            else:
                ckks_add(ctx, self.outs[z], args[0], args[1])

    def capture(self):
        """One CUDA graph per degree of the grouped schedule (after a warm run)."""
        for ln in self.ctx:
            self.run_grouped(ln)
        self.sync()
        self.graphs = {ln: Graph.capture(self.ctx[ln], lambda ln=ln: self.run_grouped(ln)) for ln in self.ctx}
        return sum(g.nodes for g in self.graphs.values())

    def launch_graphs(self):
        for ln, g in self.graphs.items():
            g.launch()

    def sync(self):
        for c in self.ctx.values():
            c.sync()


# ---------------------------------------------------------------------------------

class Server:
    """Continuous-batching request loop.  A request on ring degree 2^ln with m
    live limbs: ct * w (plaintext weights, rescaled), sum over the slots,
    rescale (the logistic-regression inner-product step).  `slots_per_degree`
    contexts (streams) per degree run requests concurrently; a request is
    admitted when its arrival time has passed, a context of its degree is free
    and the HBM budget holds its ciphertext buffers."""

    def __init__(self, log_ns=(15, 16), k=30, kl=31, slots_per_degree=4, hbm_budget=8 << 30, seed=5,
                 scale_bits=50, n_slots_used=None, autotune=False):
        rng = np.random.default_rng(seed)
        self.k, self.kl, self.log_ns = k, kl, log_ns
        primes = params.ntt_primes(60, PRIME_MODULUS, k + kl)
        self.engines, self.pool, self.keys, self.weights = {}, {}, {}, {}
        self.hbm_budget, self.hbm_used = hbm_budget, 0
        self.stats = {}
        for ln in log_ns:
            E = Engine(ln, primes[:k], primes[k:], scale_bits=scale_bits)
            if autotune:
                E.autotune()
            N = 1 << ln
            self.engines[ln] = E
            ctxs = [Context(E) for _ in range(slots_per_degree)]
            self.pool[ln] = ctxs
            # resident keys for the rotation steps 2^j and the encoded weights, shared read-only by
            # every context of the degree
            slots = n_slots_used or N // 2
            self.keys[ln] = {1 << j: SwitchKey(ctxs[0], _rand_residues(rng, primes, N), _rand_residues(rng, primes, N))
                             for j in range(int(np.log2(slots)))}
            w = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
            self.weights[ln] = ckks_encode(ctxs[0], w, empty_slots=0, scale=1 << scale_bits)[0]
            ctxs[0].sync()
        self.slots = {ln: n_slots_used or (1 << ln) // 2 for ln in log_ns}
        self.scale = 1 << scale_bits
        # resident for the server's lifetime: every degree's Galois keys (2 polys
        # of k + kl limbs each) and its encoded weights (k limbs); they count
        # against the HBM budget before any request is admitted
        self.resident_bytes = sum(len(self.keys[ln]) * 2 * (k + kl) * (1 << ln) * 8 + k * (1 << ln) * 8
                                  for ln in log_ns)

    def footprint(self, ln):
        return 3 * 2 * self.k * (1 << ln) * 8          # input, product and output ciphertexts

    def fits(self, ln):
        """Whether a request of degree 2^ln fits the HBM budget next to the
        resident keys and the requests in flight."""
        return self.resident_bytes + self.hbm_used + self.footprint(ln) <= self.hbm_budget

    def _reset_stats(self):
        self.stats = {"admitted": 0, "deferred_by_budget": 0, "deferred_by_slots": 0, "max_in_flight": 0,
                      "max_hbm_bytes": 0, "in_flight": 0}

    def _admitted(self, ln):
        st = self.stats
        st["admitted"] += 1
        st["in_flight"] += 1
        st["max_in_flight"] = max(st["max_in_flight"], st["in_flight"])
        st["max_hbm_bytes"] = max(st["max_hbm_bytes"], self.resident_bytes + self.hbm_used)

    def submit(self, ctx_index, req):
        """Enqueue a request's chain on its context (asynchronous)."""
        ln = req["log_n"]
        ctx = self.pool[ln][ctx_index]
        ct = req["ct"]
        ct.set(req["m"] - 1, self.slots[ln], self.scale, ct.domain)
        prod = req["prod"]
        ckks_mul_pt(ctx, prod, ct, self.weights[ln], self.scale, rescale=True)
        ckks_sumslots(ctx, req["out"], prod, self.keys[ln])
        ckks_rescale(ctx, req["out"])

    def run(self, requests, rate=None, poll=0.0):
        """Serve `requests` (dicts with log_n, m, ct, prod, out) arriving at
        Poisson rate `rate` per second (None: all at t = 0).  Returns per-request
        latencies (s) and the wall time."""
        import torch
        rng = np.random.default_rng(17)
        n = len(requests)
        arrivals = np.zeros(n) if rate is None else np.cumsum(rng.exponential(1.0 / rate, n))
        busy = {ln: [None] * len(self.pool[ln]) for ln in self.log_ns}
        events = {}
        pending = list(range(n))
        done_at = np.zeros(n)
        self._reset_stats()
        waited = set()
        t0 = time.perf_counter()
        remaining = n
        while remaining:
            now = time.perf_counter() - t0
            # completions
            for ln in self.log_ns:
                for i, r in enumerate(busy[ln]):
                    if r is not None and events[r].query():
                        done_at[r] = time.perf_counter() - t0
                        busy[ln][i] = None
                        self.hbm_used -= self.footprint(ln)
                        self.stats["in_flight"] -= 1
                        remaining -= 1
            # admissions (arrival order, skipping requests whose degree has no free
            # slot or that do not fit the HBM budget next to the resident keys)
            still = []
            for r in pending:
                req = requests[r]
                ln = req["log_n"]
                if arrivals[r] > now:
                    still.append(r)
                    continue
                free = [i for i, x in enumerate(busy[ln]) if x is None]
                if not free or not self.fits(ln):
                    if r not in waited:
                        waited.add(r)
                        self.stats["deferred_by_slots" if not free else "deferred_by_budget"] += 1
                    still.append(r)
                    continue
                i = free[0]
                self.submit(i, req)
                ev = torch.cuda.Event()
                ev.record(torch.cuda.ExternalStream(self.pool[ln][i].stream))
                events[r] = ev
                busy[ln][i] = r
                self.hbm_used += self.footprint(ln)
                self._admitted(ln)
            pending = still
            if poll:
                time.sleep(poll)
        wall = time.perf_counter() - t0
        return done_at - arrivals, wall

    def make_requests(self, n, seed=6, min_limbs=6, templates=None):
        """n requests (degree, live limbs, input ciphertext, product and output
        buffers).  With `templates` = t, each degree draws t distinct random
        inputs and every request gets a device copy of one of them (fast to
        make in the hundreds); otherwise every request draws its own."""
        rng = np.random.default_rng(seed)
        tmpl = {}
        if templates:
            for ln in self.log_ns:
                ctx, N, primes = self.pool[ln][0], 1 << ln, self.engines[ln].q_primes
                tmpl[ln] = [Ciphertext.from_residues(ctx, _rand_residues(rng, primes, N),
                                                     _rand_residues(rng, primes, N), slots=self.slots[ln],
                                                     scale=self.scale, domain=AOA_COEF) for _ in range(templates)]
        reqs = []
        for _ in range(n):
            ln = int(rng.choice(self.log_ns))
            m = int(rng.integers(min_limbs, self.k + 1))
            ctx = self.pool[ln][0]
            N = 1 << ln
            primes = self.engines[ln].q_primes
            if templates:
                ct = tmpl[ln][int(rng.integers(0, templates))].copy()
            else:
                ct = Ciphertext.from_residues(ctx, _rand_residues(rng, primes, N), _rand_residues(rng, primes, N),
                                              slots=self.slots[ln], scale=self.scale, domain=AOA_COEF)
            reqs.append({"log_n": ln, "m": m, "ct": ct, "prod": Ciphertext(ctx), "out": Ciphertext(ctx)})
        for c in (c for cs in self.pool.values() for c in cs):
            c.sync()
        return reqs


# ---------------------------------------------------------------------------------

class BatchServer(Server):
    """The same requests served with iteration-level batching: every
    iteration advances each active request of a ring degree by one stage of
    its chain (plaintext multiply + rescale, one rotate-and-add step of the
    slot sum, final rescale), the rotations of a stage batched over all the
    requests at that stage (aoa_rotate_batch: one key, grouped by level);
    requests that arrive join at the next iteration, finished ones leave.
    One context per degree; completion is the end of the iteration that
    finishes a request (an event on the context's stream)."""

    def __init__(self, *args, max_inflight=2, **kw):
        kw["slots_per_degree"] = 1
        super().__init__(*args, **kw)
        self.max_inflight = max_inflight

    def _steps(self, ln):
        slots = self.slots[ln]
        out, i = [], slots >> 1
        while i >= 1:
            out.append(i)
            i >>= 1
        return out

    def _iteration(self, ln, active):
        """Enqueue one stage for every active request of degree 2^ln; returns
        the requests this iteration finishes."""
        ctx = self.pool[ln][0]
        steps = self._steps(ln)
        by_stage = {}
        for r in active:
            by_stage.setdefault(r["stage"], []).append(r)
        done = []
        for stage, reqs in by_stage.items():
            if stage == 0:
                for r in reqs:
                    ct = r["ct"]
                    ct.set(r["m"] - 1, self.slots[ln], self.scale, ct.domain)
                    ckks_mul_pt(ctx, r["out"], ct, self.weights[ln], self.scale, rescale=True)
            elif stage <= len(steps):
                step = steps[stage - 1]
                ckks_rotate_batch(ctx, [r["prod"] for r in reqs], [r["out"] for r in reqs], step,
                                  self.keys[ln][step])
                for r in reqs:
                    ckks_add(ctx, r["out"], r["out"], r["prod"])
            else:
                for r in reqs:
                    ckks_rescale(ctx, r["out"])
                    done.append(r)
            for r in reqs:
                r["stage"] += 1
        return done

    def submit(self, ctx_index, req):
        """Run one request alone through the same stages."""
        ln = req["log_n"]
        req["stage"] = 0
        while req["stage"] <= len(self._steps(ln)) + 1:
            self._iteration(ln, [req])

    def run(self, requests, rate=None, poll=0.0):
        import torch
        rng = np.random.default_rng(17)
        n = len(requests)
        arrivals = np.zeros(n) if rate is None else np.cumsum(rng.exponential(1.0 / rate, n))
        for r in requests:
            r["stage"] = 0
        active = {ln: [] for ln in self.log_ns}
        inflight = {ln: [] for ln in self.log_ns}        # (event, finished request ids)
        pending = list(range(n))
        done_at = np.zeros(n)
        ids = {id(r): i for i, r in enumerate(requests)}
        self._reset_stats()
        waited = set()
        t0 = time.perf_counter()
        remaining = n
        while remaining:
            now = time.perf_counter() - t0
            for ln in self.log_ns:                          # completions
                keep = []
                for ev, fin in inflight[ln]:
                    if ev.query():
                        t = time.perf_counter() - t0
                        for i in fin:
                            done_at[i] = t
                            remaining -= 1
                            self.hbm_used -= self.footprint(ln)
                            self.stats["in_flight"] -= 1
                    else:
                        keep.append((ev, fin))
                inflight[ln] = keep
            still = []
            for i in pending:                               # admissions: the HBM budget binds
                r = requests[i]
                ln = r["log_n"]
                if arrivals[i] > now:
                    still.append(i)
                    continue
                if not self.fits(ln):
                    if i not in waited:
                        waited.add(i)
                        self.stats["deferred_by_budget"] += 1
                    still.append(i)
                    continue
                active[ln].append(r)
                self.hbm_used += self.footprint(ln)
                self._admitted(ln)
            pending = still
            for ln in self.log_ns:                          # one iteration per degree
                if not active[ln] or len(inflight[ln]) >= self.max_inflight:
                    continue
                fin = self._iteration(ln, active[ln])
                ev = torch.cuda.Event()
                ev.record(torch.cuda.ExternalStream(self.pool[ln][0].stream))
                inflight[ln].append((ev, [ids[id(r)] for r in fin]))
                finished = {id(r) for r in fin}
                active[ln] = [r for r in active[ln] if id(r) not in finished]
            if poll:
                time.sleep(poll)
        wall = time.perf_counter() - t0
        return done_at - arrivals, wall
