"""Benchmark of the tet4 ADER-DG element update on B200.

One step = one GTS time step (local -> sources -> neighbour, with receiver sampling) over the whole
mesh and all fused runs. Default workload (the headline configuration): a 10 km box of 48^3 cubes
x 6 tets (663,552 tets), ORDER 5 (35 modes), 16 fused runs in FP32, homogeneous material
(vp 6000, vs 3464, rho 2670), one seeded random point source per run (moment tensor N(0,1) x 1e15,
1.5 Hz Ricker), 8 receivers, free surface on top and outflow elsewhere. Inputs are synthetic.

Prints one JSON line (rank 0). ``--impl reference`` times the reference's own CPU kernels
(compiled from its sources into oracle/_ref; the oracle port if that build is absent) on the host.
Multi-GPU: replicas only (every rank runs the full workload; no data-path collective).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "elastic element-updates/s: batched FP32 vs plain FP64 at rel-L2 1e-4; p50/p99"
UNIT = "element-updates/s"

from edge_b200.workloads import WORKLOADS  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="edge", choices=["edge", "reference"])
    ap.add_argument("--workload", default="box48_o5_r16_fp32", choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--tc-probe", action=argparse.BooleanOptionalAction, default=True,
                    help="time tcgen05 tf32 MMAs at the DG products' shapes (the tensor-core alternative)")
    ap.add_argument("--parity", action=argparse.BooleanOptionalAction, default=True,
                    help="per-run FP32 receiver error against FP64 at the workload's full size and steps")
    ap.add_argument("--serve-requests", type=int, default=160,
                    help="requests of the serving run (Poisson arrivals); 0 skips it")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="mean arrivals per second")
    ap.add_argument("--lts-report", action=argparse.BooleanOptionalAction, default=True,
                    help="also time rate-2 LTS against GTS on a layered box")
    ap.add_argument("--batch-sims", type=int, default=64,
                    help="simulations of the uneven-batch run (graph-captured batch steps); 0 skips it")
    return ap.parse_args()


def dist_init(n_gpus):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """Samples nvidia-smi while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_problem(name):
    from edge_b200 import workloads
    prob, w = workloads.build(name)
    return prob, w.precision


def host_n_modes(order):
    return order * (order + 1) * (order + 2) // 6


def algorithmic(prob, prec, premix=False, fs_pair=84, fused=False, char=False):
    """Per-element algorithmic bytes and flops of one step (dense-in-modes counts as in the
    roofline model of the path) for each kernel. premix: the local kernel mixes the face
    projections with the reading element's flux solver and reads per face the padded pair
    [2][fs_pair] of flux solvers in the compute precision instead of its own fsE[0] block; the
    neighbour kernel then reads no flux solvers. char: the local kernel mixes through the rank-3
    factors of each face's flux-solver pair (3 x 9 + 2 x 9 x 3 products per face mode for both
    mixes instead of 2 x 81) and reads 108 factor values per face instead of the pair. fused: the
    local kernel also runs the previous step's neighbour step (reads the four neighbour projections
    and the connectivity, adds their lifted fluxes and stores the completed DOF rows once more)."""
    from edge_b200.host import n_face_modes, n_modes
    O, R, rm = prob.order, prob.runs, prob.rm
    B, F, p = n_modes(O), n_face_modes(O), (8 if prec == 64 else 4)
    Bm = lambda o: n_modes(o) if o > 0 else 0
    ck = sum(3 * (2 * 9 * Bm(O - d) * Bm(O - d + 1) + 2 * 24 * Bm(O - d)) + 2 * 9 * Bm(O - d) for d in range(1, O))
    vol = 3 * (2 * 9 * B * Bm(O - 1) + 2 * 24 * B)
    surf = 4 * (2 * 9 * F * B + 2 * 81 * F + 2 * 9 * B * F)
    dofs = (9 + 6 * rm) * B * R * p
    face = 4 * 9 * F * R * p
    fs_local = 4 * 108 * p if char else (4 * 2 * fs_pair * p if premix else 4 * 81 * 8)
    local_bytes = 2 * dofs + face + 3 * 24 * 8 + fs_local + (rm * 12 * 8 + 27 * 8 + 4 * 54 * 8 if rm else 0)
    neigh_bytes = 2 * dofs + face + (0 if premix else 4 * 81 * 8) + 4 * (4 + 1 + 1 + 1) + (4 * 54 * 8 if rm else 0)
    # the face mixes: surf counts one 9 x 9 mix per face; pre-mixing adds the second, and the
    # factors replace both by 3 x 9 + 2 x 9 x 3 products per face mode
    mix = (4 * 2 * (81 + 54 - 2 * 81) * F if char else 0) + (4 * 2 * 81 * F if premix else 0)
    local_flops = (ck + vol + surf + mix) * R
    neigh_flops = (surf - 4 * 2 * 81 * F) * R if premix else surf * R
    if fused:
        local_bytes += face + dofs + 4 * (4 + 1 + 1 + 1)
        local_flops += neigh_flops
    return dict(local_bytes=local_bytes, neigh_bytes=neigh_bytes, local_flops=local_flops, neigh_flops=neigh_flops)


def compulsory_step_bytes(prob, prec):
    """Compulsory bytes of one element step with every array touched once: DOFs (elastic and
    anelastic) read and written, the time-integrated DOFs written and read once, the FP64 star
    matrices (3 x 24), both flux-solver sets (2 x 4 x 81) and, with attenuation, the anelastic
    sources, star matrices and flux solvers, plus 24 bytes of connectivity."""
    from edge_b200.host import n_modes
    B, R, rm, p = n_modes(prob.order), prob.runs, prob.rm, (8 if prec == 64 else 4)
    b = 2 * (9 + 6 * rm) * B * R * p + 2 * 9 * B * R * p + 3 * 24 * 8 + 2 * 4 * 81 * 8 + 24
    if rm:
        b += 12 * 8 * rm + 3 * 9 * 8 + 2 * 4 * 54 * 8
    return b


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d["hbm_gbs"], "of measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "of fallback"


def peak_clock_mhz():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["sm_max_mhz"])
    except (OSError, KeyError, ValueError):
        return 1965.0


def traffic_from_profiles(workload):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"kLocal_{workload}.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_full_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def cpu_reference_rate(order, runs, rm, n_cubes=16, steps=3, warm=1, r1=True):
    """The reference's own vanilla CPU kernels (oracle/_ref, OpenMP over all host threads) on a
    bounded sample of the workload: a box of n_cubes^3 x 6 tets (16^3: 24,576 tets; FP64 DOFs and
    time-integrated DOFs of 2 x 9 x B x R x 8 bytes per element, 2.2 GB at order 5 with 16 runs,
    beyond any L3), with its mesh and elastic element data built by the oracle's numpy mesh code
    and the reference's compiled Elasticity::star / ::fs. `warm` untimed steps (the first constructs
    the kernels), then the median of `steps` timed steps (local + neighbour). With r1, the same
    sample is also timed with the one-run build, the rate of running the R runs one after another.
    Falls back to the C oracle port (one thread) where oracle/_ref is absent.
    Returns (element-updates/s, kind, cores, sample text, extra dict)."""
    import numpy as np
    for p in (os.path.join(ROOT, "oracle"),):
        if p not in sys.path:
            sys.path.insert(0, p)
    import mesh as om
    import oracle as orc
    import ref as refmod
    L = refmod.load(order, runs, rm)
    m = om.box(n_cubes)
    ne = m["n_el"]
    rho = np.full(ne, 2670.0)
    mu = rho * 3464.0 ** 2
    lam = rho * 6000.0 ** 2 - 2 * mu
    extra = {}
    setup = "mesh: oracle numpy box; element data: reference Elasticity::star/fs"
    if L is not None:
        starE, fsE = om.elastic_data(L, m, rho, lam, mu)
    else:
        from edge_b200 import host
        hm = host.Mesh.box(n_cubes)
        starE, fsE = host.star(hm, rho, lam, mu), host.flux_solvers(hm, rho, lam, mu)[0]
        setup = "mesh and element data: host setup (oracle/_ref absent)"
    d = dict(order=order, runs=runs, rm=rm, nEl=ne, starE=starE, fsE=fsE, elFaEl=m["el_fa_el"],
             fIdElFaEl=m["fid"], vIdElFaEl=m["vid"], faType=m["el_fa_type"], starA=None, srcA=None, fsA=None,
             omega=None)
    if rm:
        # anelastic coefficients through the host setup (the reference's needs Eigen, absent here)
        from edge_b200 import host
        hm = host.Mesh.box(n_cubes)
        rng = np.random.default_rng(3343)
        d["srcA"], d["omega"], lam2, mu2 = host.attenuation(rm, 1.0, 100.0, rng.uniform(50, 200, ne),
                                                            rng.uniform(50, 200, ne), lam.copy(), mu.copy())
        d["starA"] = host.star_anelastic(hm)
        d["fsA"] = host.flux_solvers(hm, rho, lam2, mu2, rm)[1]
        setup += "; anelastic data: host setup"
    from edge_b200.dgmat import matrices
    d.update({k: v for k, v in matrices(order).items() if k in ("stiffT", "stiffV", "fluxL", "fluxN", "fluxT")})
    d = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    dt = 0.5 * float(m["el_india"].min()) / 6000.0 / (2 * order - 1)
    B = host_n_modes(order)
    rng = np.random.default_rng(0)

    def state(r):
        return dict(dofsE=rng.normal(size=(ne, 9, B, r)), dofsA=rng.normal(size=(ne, rm, 6, B, r)) if rm else None,
                    tDofs=np.zeros((ne, 9, B, r)))

    def timed(lib, r, n_warm, n_timed):
        st = state(r)
        dd = dict(d, runs=r)
        ts = []
        for i in range(n_warm + n_timed):
            t0 = time.perf_counter()
            if lib is not None:
                refmod.step(lib, dd, st, 0.0, dt)
            else:
                orc.step(dd, st, 0.0, dt)
            if i >= n_warm:
                ts.append(time.perf_counter() - t0)
        return ne * r / statistics.median(ts), ts

    cores = os.cpu_count() or 1
    kind = "reference" if L is not None else "port"
    if L is None:
        cores = 1
    value, ts = timed(L, runs, warm, steps)
    sample = (f"{n_cubes}^3 cubes x 6 = {ne} tets, order {order}, {runs} runs, {rm} mechanisms, FP64, "
              f"{warm} warm-up + median of {steps} timed steps (local + neighbour); {setup}")
    extra["step_s"] = ts
    if r1 and runs > 1:
        L1 = refmod.load(order, 1, rm)
        if L1 is not None:
            v1, t1 = timed(L1, 1, 1, max(steps, 3))
            extra["one_run_build"] = {"value": v1, "unit": UNIT, "step_s": t1,
                                      "note": f"the {runs} runs one after another with the one-run build"}
    return value, kind, cores, sample, extra


# the serving stream: four seeded meshes with their material sets (10,368 to 1,053,696 tets), the
# orders each serves (elastic; viscoelastic requests at orders 3-4 where listed) and the step range
# of its requests
SERVE_MESHES = {
    "box12": (dict(n_cubes=12, ext=7.5e3, seed=11), (3, 4, 5, 6), (3, 4), (200, 2000)),
    "box20j": (dict(n_cubes=20, jitter=0.1, layers=(4000.0, 5500.0, 6500.0), lognormal_sigma=0.1, seed=12),
               (3, 4, 5, 6), (3, 4), (100, 1000)),
    "box32": (dict(n_cubes=32, layers=(4000.0, 6000.0), lognormal_sigma=0.1, seed=13), (3, 4, 5, 6), (3, 4),
              (100, 400)),
    "box56": (dict(n_cubes=56, seed=14), (3, 4, 5, 6), (), (100, 150)),
}


def serve_stream(n_req, rate, seed):
    """Requests of the bounded serving stream: Poisson(rate) arrivals over SERVE_MESHES, 25%
    viscoelastic where the mesh serves it, 4-16 receivers, the mesh's step range."""
    import numpy as np
    from edge_b200 import serve
    specs = {k: serve.MeshSpec(**v[0]) for k, v in SERVE_MESHES.items()}
    rng = np.random.default_rng(seed)
    reqs = serve.make_stream(n_req, rate, specs, orders=(3, 4, 5, 6), seed=seed, visco=0.25,
                             mesh_steps={k: v[3] for k, v in SERVE_MESHES.items()})
    for r in reqs:  # each mesh's own orders and physics
        _, orders, vorders, _ = SERVE_MESHES[r.mesh]
        if r.rm and not vorders:
            r.rm = 0
        allowed = vorders if r.rm else orders
        if r.order not in allowed:
            r.order = int(rng.choice(allowed))
    return specs, reqs


def run_serve(n_req, rate, device, seed=3343, n_check=12):
    """The serving form on a bounded stream shaped like the serving configuration: n_req requests
    (Poisson arrivals at `rate` per second) over four meshes of 10,368 to 1,053,696 tets with
    their own material sets, orders 3-6 (elastic) and 3-4 (viscoelastic, 3 mechanisms), 100-2,000
    steps, 4-16 receivers and own random sources, continuously batched into 16-run FP32 pools under
    an 80% HBM budget. Two passes over the same seeded requests: all arriving at once (capacity:
    delivered element updates per second against running each request alone as a plain FP64
    single run, timed per mesh / order / physics on the same GPU) and the Poisson stream (latency
    percentiles). Pools take 1, 4, 8 or 16 fused runs as the waiting requests and the HBM budget
    allow (the 1 M-tet mesh at orders 5-6 fits 4-8 runs). n_check requests (spread over meshes and
    physics) are run again alone on the plain FP64 path and their served receiver traces compared
    by relative L2."""
    import numpy as np
    import torch
    from edge_b200 import serve
    from edge_b200.solver import Solver
    out = {}
    specs, reqs0 = serve_stream(n_req, rate, seed)
    keys = sorted({(r.mesh, r.order, r.rm) for r in reqs0})
    meshes = serve.MeshCache(specs)
    for k in keys:  # host setup of every mesh, material set and physics outside the timed passes
        meshes.data(k[0], k[2])
    served = None
    for name, r8 in (("burst", None), ("poisson", rate)):
        _, reqs = serve_stream(n_req, rate, seed)
        if r8 is None:
            for r in reqs:
                r.arrival = 0.0
        srv = serve.Server(specs, runs=16, precision=32, chunk=40, device=device)
        srv.meshes = meshes
        done = srv.run(reqs, clock="wall")
        srv.close()
        lat = serve.latency_stats(done)
        n_el = {k: meshes.data(k, 0)["mesh"].n_el for k in specs}
        out[name] = dict(requests=len(done), arrival_rate_per_s=r8, wall_s=srv.wall, latency_s_p50=lat["p50"],
                         latency_s_p99=lat["p99"], pools_opened=srv.pools_opened, max_pools=srv.max_pools,
                         pool_resizes=srv.resizes,
                         slot_utilisation=srv.slot_updates_used / max(srv.slot_updates_offered, 1),
                         delivered_element_updates_per_s=sum(n_el[x.mesh] * x.n_steps for x in done) / srv.wall)
        if name == "burst":
            served = {x.rid: x for x in done}
    # plain FP64, one run, same mesh, order and physics: ms per step
    ms64 = {}
    for m, o, rm in keys:
        p = meshes.problem(m, o, 1, rm)
        st = torch.cuda.Stream(device=device)
        sv = Solver(p, precision=64, stream=st.cuda_stream, device=device)
        e, a = p.zero_dofs()
        sv.upload_dofs(e, a)
        sv.step(3)
        sv.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sv.step(20)
        e1.record(st)
        torch.cuda.synchronize()
        ms64[(m, o, rm)] = e0.elapsed_time(e1) / 20
        sv.close()
    # the same keys as 16-run FP32 pools at full occupancy (8 runs where 16 exceed the budget: the
    # kernel-level ratio the serving form can reach), and the cost of opening such a pool
    ms32, open_s, runs32 = {}, {}, {}
    budget = 0.8 * torch.cuda.mem_get_info(device)[1]
    for m, o, rm in keys:
        t_open = time.perf_counter()
        nr = 16 if serve.pool_bytes(meshes.data(m, rm)["mesh"].n_el, o, 16, 32, rm) < budget else 8
        runs32[(m, o, rm)] = nr
        p = meshes.problem(m, o, nr, rm)
        st = torch.cuda.Stream(device=device)
        sv = Solver(p, precision=32, stream=st.cuda_stream, device=device)
        sv.step(3)
        sv.sync()
        open_s[(m, o, rm)] = time.perf_counter() - t_open
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sv.step(20)
        e1.record(st)
        torch.cuda.synchronize()
        ms32[(m, o, rm)] = e0.elapsed_time(e1) / 20 * 16 / nr  # per 16 runs
        sv.close()
    serial_s = sum(ms64[(x.mesh, x.order, x.rm)] * x.n_steps for x in reqs0) / 1e3
    ideal_s = sum(ms32[(x.mesh, x.order, x.rm)] / 16 * x.n_steps for x in reqs0) / 1e3
    out["burst"]["serial_plain_fp64_s"] = serial_s
    out["burst"]["speedup_vs_serial_plain_fp64"] = serial_s / out["burst"]["wall_s"]
    out["burst"]["full_pools_fp32_s"] = ideal_s
    out["burst"]["kernel_level_speedup"] = serial_s / ideal_s
    # per-request error of served results against the plain FP64 path
    rng = np.random.default_rng(seed + 1)
    groups = {}
    for x in reqs0:
        groups.setdefault((x.mesh, x.rm), []).append(x.rid)
    pick = []
    while len(pick) < n_check and any(groups.values()):
        for g in sorted(groups):
            if groups[g] and len(pick) < n_check:
                pick.append(groups[g].pop(int(rng.integers(len(groups[g])))))
    checks = []
    for rid in pick:
        x = served[rid]
        ref = serve.plain_fp64(x, meshes, device=device)
        got = x.result()
        checks.append(dict(rid=rid, mesh=x.mesh, order=x.order, mechanisms=x.rm, steps=x.n_steps,
                           receivers=len(x.rec_pos),
                           rel_l2=float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-300))))
    out.update(pools=len(keys), slots_per_pool=16, chunk_steps=40,
               meshes={k: meshes.data(k, 0)["mesh"].n_el for k in specs},
               stream=dict(requests=n_req, rate_per_s=rate, viscoelastic=sum(1 for x in reqs0 if x.rm),
                           orders=sorted({x.order for x in reqs0}),
                           steps=[min(x.n_steps for x in reqs0), max(x.n_steps for x in reqs0)]),
               per_request_fp64_check=checks, per_request_rel_l2_max=max(c["rel_l2"] for c in checks),
               plain_fp64_ms_per_step={f"{m}/o{o}/m{rm}": v for (m, o, rm), v in ms64.items()},
               fp32_16runs_ms_per_step={f"{m}/o{o}/m{rm}": v for (m, o, rm), v in ms32.items()},
               pool_open_s={f"{m}/o{o}/m{rm}": v for (m, o, rm), v in open_s.items()},
               note="wall clock from the first arrival; latency = arrival -> last receiver sample on the host; "
                    "bounded stream (the 2,000-request, 2 M-tet configuration does not fit one run of the bench: "
                    "16-run pools of 2 M tets at order 6 need about 430 GB)")
    return out


def run_tc_probe(local_ms, n_el, order, runs, device, clock_mhz):
    """The tensor-core alternative for the local kernel's DG products, measured: tcgen05.mma
    (kind::tf32, and kind::f16 with bf16 operands; operands in shared memory, accumulator in tensor
    memory) timed per instruction of 128 x N x K (K = 8 tf32, 16 bf16) for the N the products would
    have, with one and two issuing CTAs per SM, then the instructions one local step needs in the
    tensor formulation -- rows (quantity, element, run) on M in tiles of 128 (the 288 rows of an
    element group in three tiles), output modes on N (padded to 16), input modes x 3 derivative
    directions (or x 4 faces) on K, each product three times for FP32-level accuracy (split
    operands: 3xtf32 or 3xbf16) -- at the measured cycles. Only the products: the star and
    flux-solver mixes, the operand splits, loads, stores and tensor-memory read-back come on top."""
    from edge_b200 import tcprobe
    from edge_b200.host import n_face_modes, n_modes
    errs = {f"{kind}_{n}x{k}x{it}": tcprobe.check(n, k, it, kind=kind)
            for kind, n, k, it in (("tf32", 16, 8, 1), ("tf32", 64, 32, 1), ("tf32", 128, 32, 3),
                                   ("bf16", 16, 16, 1), ("bf16", 128, 64, 3))}
    ns = (16, 32, 48, 64, 96, 128)

    def cycles(kind, acc, per_sm):
        # cycles per instruction of one SM; two CTAs per SM only where their tensor memory fits
        out = {}
        for n in ns:
            if per_sm == 2 and acc == 3 and n > 64:
                continue
            ms, per_sm_instr = tcprobe.time_shape(n, acc=acc, kind=kind, per_sm=per_sm)
            out[n] = ms * 1e-3 * clock_mhz * 1e6 / per_sm_instr
        return out

    meas = {"tf32_acc1": cycles("tf32", 1, 1), "tf32_acc3": cycles("tf32", 3, 1),
            "tf32_acc3_2cta": cycles("tf32", 3, 2), "bf16_acc3": cycles("bf16", 3, 1),
            "bf16_acc3_2cta": cycles("bf16", 3, 2)}
    pad = lambda x, q: (x + q - 1) // q * q
    Bm = lambda o: n_modes(o) if o > 0 else 0
    F = n_face_modes(order)
    prods = [("ck%d" % d, pad(Bm(order - d), 16), 3 * Bm(order - d + 1)) for d in range(1, order)]
    prods += [("volume", pad(Bm(order), 16), 3 * Bm(order - 1)), ("fluxL", pad(4 * F, 16), Bm(order)),
              ("fluxT", pad(Bm(order), 16), 4 * F)]
    groups_per_sm = n_el * runs / 32 / 148
    tiles, split = 3, 3

    def estimate(kind, cyc, cyc_wide):
        kq = tcprobe.K_INSTR[kind]
        est = {}
        for name, nn, kk in prods:
            table = cyc if nn in cyc else cyc_wide  # N beyond the two-CTA range: one CTA per SM
            c = table[min(x for x in table if x >= nn)]
            est[name] = groups_per_sm * tiles * split * (pad(kk, kq) // kq) * c / (clock_mhz * 1e3)
        return est

    options = {"3xtf32": estimate("tf32", meas["tf32_acc3"], meas["tf32_acc3"]),
               "3xtf32_2cta": estimate("tf32", meas["tf32_acc3_2cta"], meas["tf32_acc3"]),
               "3xbf16": estimate("bf16", meas["bf16_acc3"], meas["bf16_acc3"]),
               "3xbf16_2cta": estimate("bf16", meas["bf16_acc3_2cta"], meas["bf16_acc3"])}
    totals = {k: sum(v.values()) for k, v in options.items()}
    best = min(totals, key=totals.get)
    return {"check_rel_err": errs, "cycles_per_instruction_per_sm_128xNxK": meas, "clock_mhz": clock_mhz,
            "products": [{"name": a, "N": b, "K": c} for a, b, c in prods],
            "tensor_ms_per_step_by_product": options, "tensor_ms_per_step": totals, "best": best,
            "fused_local_kernel_ms": local_ms, "ratio_best_tensor_products_to_whole_fp32_kernel": totals[best] / local_ms,
            "note": "split-operand products only, at the measured per-instruction rate; the FP32 kernel's time "
                    "includes everything"}


# FP32 configurations the uneven batch draws from: orders 3-6, fused runs 1 / 4 / 8 / 16, elastic
# or 3 mechanisms (order, runs, mechanisms)
BATCH_CFGS = [(o, r, rm) for o in (3, 4, 5, 6) for r in (1, 4, 8, 16) for rm in (0, 3)]
# four seeded boxes of the batch configuration's sizes: (cubes per axis, vertex jitter)
BATCH_BOXES = [(10, 0.0), (19, 0.05), (29, 0.1), (44, 0.2)]


def _batch_sims(n_sims, seed, step_range):
    """The seeded simulations of the uneven batch: (mesh index, order, runs, mechanisms, steps)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_sims):
        mi = int(rng.integers(len(BATCH_BOXES)))
        o, r, rm = BATCH_CFGS[int(rng.integers(len(BATCH_CFGS)))]
        out.append((mi, o, r, rm, int(rng.integers(step_range[0], step_range[1] + 1))))
    return out


def run_batch(n_sims, device, seed=3343, mem_fraction=0.6, step_range=(20, 100)):
    """The uneven batch configuration: n_sims simulations over four seeded boxes of 6,000, 41,154,
    146,334 and 511,104 tets (jitter 0 / 5 / 10 / 20%), each with its own order (3-6), fused runs
    (1, 4, 8, 16), physics (elastic or 3 mechanisms), random sources and step count (step_range; the
    configuration's 200-1000 steps scaled by 1/10 to bound the run). Simulations are admitted in
    waves by an HBM budget (mem_fraction of the free memory). Every wave runs three ways, timed on the
    wall clock after a device sync: each simulation alone after another (its own fused multi-step
    calls), the graph-captured batch steps of edge_b200_batch_* (a stream per context), and the
    merged form (edge_b200.merged: one context and one persistent launch per kernel and step for
    each configuration family, the families on streams of their own). Also against each simulation
    alone on the plain FP64 path (one run per fused run; FP64 ms per step measured per mesh, order and
    physics; viscoelastic orders 5-6 have no FP64 path and are left out of that sum)."""
    import time

    import numpy as np
    import torch
    from edge_b200 import host
    from edge_b200.batch import Batch
    from edge_b200.merged import MergedFamily, family_key
    from edge_b200.solver import Solver
    meshes = [host.Mesh.box(n, (1e4, 1e4, 1e4), jitter=j, seed=seed + i) for i, (n, j) in enumerate(BATCH_BOXES)]
    base = {}

    def elem(mi, rm):
        if (mi, rm) not in base:
            m = meshes[mi]
            rng = np.random.default_rng(seed + 7 * mi + rm)
            rho, lam, mu = host.materials(m, 1e4, rng=rng)
            qp = rng.uniform(50.0, 200.0, m.n_el) if rm else None
            qs = rng.uniform(50.0, 200.0, m.n_el) if rm else None
            base[(mi, rm)] = (rho, host.element_data(m, rho, lam, mu, rm, qp, qs))
        return base[(mi, rm)]

    def problem(k, mi, o, r, rm, steps):
        rho, d = elem(mi, rm)
        m = meshes[mi]
        dt = host.dt_cfl(m, o, rho, d["lam"], d["mu"])
        rng = np.random.default_rng(seed + 17 * k)
        pos = rng.uniform(1e3, 9e3, (r, 3))
        scal = np.concatenate([rng.normal(0.0, 1.0, (r, 6)) * 1e15, np.zeros((r, 3))], axis=1)
        dts = dt / 10.0
        src = host.make_sources(m, o, r, pos, scal, 1.5, 0.8, dts, int(np.ceil(steps * dt / dts)) + 4)
        return host.Problem(order=o, runs=r, rm=rm, mesh=m, rho=rho, lam=d["lam"], mu=d["mu"], starE=d["starE"],
                            fsE=d["fsE"], dt=dt, starA=d["starA"], srcA=d["srcA"], fsA=d["fsA"], omega=d["omega"],
                            sources=src, name=f"sim{k}")

    sims = _batch_sims(n_sims, seed, step_range)
    budget = torch.cuda.mem_get_info(device)[0] * mem_fraction
    waves, cur, used = [], [], 0.0
    for k, (mi, o, r, rm, steps) in enumerate(sims):
        B, F = host.n_modes(o), o * (o + 1) // 2
        need = meshes[mi].n_el * (r * 4 * ((9 + 6 * rm) * (B + 4) * 3 + 2 * 36 * (F + 4)) + 8000)
        if cur and used + need > budget:
            waves.append(cur)
            cur, used = [], 0.0
        cur.append(k)
        used += need
    if cur:
        waves.append(cur)
    t_seq = t_batch = t_merged = 0.0
    upd = 0
    merged_launches = seq_launches = 0
    fams_total = 0
    for wave in waves:
        probs = {k: problem(k, *sims[k]) for k in wave}
        steps = [sims[k][4] for k in wave]
        upd += sum(probs[k].n_el * sims[k][2] * sims[k][4] for k in wave)
        solvers = []
        for k in wave:
            sv = Solver(probs[k], precision=32, device=device)
            e0, a0 = probs[k].zero_dofs(np.float32)
            sv.upload_dofs(e0, a0)
            sv.step(1)  # per-context setup (flux-solver factors, buffers) outside the timing
            solvers.append(sv)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for sv, n in zip(solvers, steps):
            sv.step(n)
            seq_launches += sv.launches()
        torch.cuda.synchronize()
        t_seq += time.perf_counter() - t0
        b = Batch(solvers, autotune=False)
        b.run(1)  # captures the graph once outside the timing
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run(steps)
        t_batch += time.perf_counter() - t0
        b.close()
        for sv in solvers:
            sv.close()
        del solvers
        # merged families, each on a stream of its own
        fams = {}
        for k in wave:
            fams.setdefault(family_key(probs[k], 32), []).append(k)
        objs = []
        for key, ks in fams.items():
            st = torch.cuda.Stream(device=device)
            fam = MergedFamily([probs[k] for k in ks], [sims[k][4] for k in ks], precision=32, device=device,
                               stream=st.cuda_stream)
            fam.solver.step(1)  # setup outside the timing, as for the others
            objs.append((fam, st))
        fams_total += len(objs)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for fam, _ in objs:
            merged_launches += fam.launch()
        torch.cuda.synchronize()
        t_merged += time.perf_counter() - t0
        for fam, _ in objs:
            fam.close()
        del objs
    # plain FP64, one run: ms per step per (mesh, order, mechanisms)
    ms64 = {}
    for k, (mi, o, r, rm, n) in enumerate(sims):
        key = (mi, o, rm)
        if key in ms64 or (rm and o > 4):
            continue
        p = problem(k, mi, o, 1, rm, 4)
        p.sources = {}
        s64 = Solver(p, precision=64, device=device)
        s64.step(2)
        s64.sync()
        t1 = time.perf_counter()
        s64.step(10)
        s64.sync()
        ms64[key] = (time.perf_counter() - t1) / 10 * 1e3
        s64.close()
    # one configuration family of many small simulations (the case merging is for): 32 simulations
    # of order 4, 8 runs, elastic on the 6,000-tet box with their own sources and the configuration's
    # 200-1,000 steps, alone after another against one merged context (each side set up by one
    # untimed step first)
    fam_sims = [(0, 4, 8, 0, int(n)) for n in np.random.default_rng(seed + 5).integers(200, 1001, 32)]
    fprobs = [problem(1000 + k, *x) for k, x in enumerate(fam_sims)]
    fsteps = [x[4] for x in fam_sims]
    fupd = sum(p.n_el * 8 * n for p, n in zip(fprobs, fsteps))
    solvers = []
    for p in fprobs:
        sv = Solver(p, precision=32, device=device)
        e0, _ = p.zero_dofs(np.float32)
        sv.upload_dofs(e0)
        sv.step(1)
        solvers.append(sv)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for sv, n in zip(solvers, fsteps):
        sv.step(n)
    torch.cuda.synchronize()
    f_seq = time.perf_counter() - t0
    for sv in solvers:
        sv.close()
    fam = MergedFamily(fprobs, fsteps, precision=32, device=device)
    fam.solver.step(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fam.launch()
    torch.cuda.synchronize()
    f_merged = time.perf_counter() - t0
    fam.close()
    small_family = {"simulations": len(fam_sims), "tets": fprobs[0].n_el, "order": 4, "runs": 8,
                    "element_updates": fupd, "one_after_another_fp32_s": f_seq, "merged_s": f_merged,
                    "speedup_vs_one_after_another_fp32": f_seq / f_merged}
    have64 = [x for x in sims if (x[0], x[1], x[3]) in ms64]
    t64 = sum(ms64[(mi, o, rm)] * r * n for mi, o, r, rm, n in have64) / 1e3
    frac64 = sum(meshes[x[0]].n_el * x[2] * x[4] for x in have64) / max(upd, 1)
    return {"simulations": len(sims), "waves": len(waves), "tets": [m.n_el for m in meshes],
            "configs": sorted({(o, r, rm) for _, o, r, rm, _ in sims}), "configuration_families": fams_total,
            "steps_range": list(step_range), "element_updates": upd,
            "one_after_another_fp32_s": t_seq, "graph_batch_s": t_batch, "merged_s": t_merged,
            "element_updates_per_s": upd / t_merged,
            "speedup_vs_one_after_another_fp32": t_seq / t_merged,
            "graph_batch_speedup_vs_one_after_another_fp32": t_seq / t_batch,
            "kernel_launches": {"one_after_another": seq_launches, "merged": merged_launches},
            "plain_fp64_alone_s_covered": t64, "fp64_covered_fraction_of_updates": frac64,
            "speedup_vs_plain_fp64_alone": t64 / (t_merged * frac64) if frac64 > 0 else None,
            "small_family": small_family,
            "note": "wall clock (host timer after a device sync); the FP64 comparison covers the simulations "
                    "with an FP64 configuration and scales the merged time by their share of the updates"}


def run_lts(device, n_cubes=48, order=5, runs=16, n_groups=3, cycles=2):
    """Rate-2 LTS against GTS on a layered box (vp 1500 / 3000 / 6000 m/s from the top, free surface
    on top): elements sorted into EDGE-V time groups; both advance the same simulated time (GTS at
    the fundamental step). Reports the element updates each performs per second of wall time and
    the wall-time ratio."""
    import numpy as np
    import torch
    from edge_b200 import host
    from edge_b200.solver import Solver
    layers = [1500.0, 3000.0, 6000.0]
    base = host.build_problem(n_cubes, order, runs, layers=layers, seed=3343, source="random", n_receivers=8,
                              n_steps=64)
    dt_el = host.dt_cfl_el(base.mesh, order, base.rho, base.lam, base.mu)
    tg = host.time_groups(base.mesh, dt_el, n_groups)
    mesh, perm, gf = host.sort_by_groups(base.mesh, tg)
    prob = host.build_problem(n_cubes, order, runs, layers=layers, seed=3343, source="random", n_receivers=8,
                              n_steps=64, mesh=mesh)
    counts = np.diff(gf)
    n_fun = cycles * (1 << (n_groups - 1))
    st = torch.cuda.Stream(device=device)
    out = {"tets": prob.n_el, "order": order, "runs": runs, "groups": counts.tolist(),
           "fundamental_steps": n_fun}
    for mode in ("gts", "lts"):
        s = Solver(prob, precision=32, stream=st.cuda_stream, device=device)
        s.upload_dofs(prob.zero_dofs(np.float32)[0])
        if mode == "lts":
            s.set_time_groups(gf)
            s.step_lts(1)
        else:
            s.step(2)
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        if mode == "lts":
            s.step_lts(cycles)
        else:
            s.step(n_fun)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        s.close()
        upd = (sum(int(c) * (n_fun >> g) for g, c in enumerate(counts)) if mode == "lts" else prob.n_el * n_fun)
        out[mode] = {"ms": ms, "element_updates_per_s": upd * runs / (ms / 1e3),
                     "gts_equivalent_element_updates_per_s": prob.n_el * n_fun * runs / (ms / 1e3)}
    out["speedup_lts_over_gts"] = out["gts"]["ms"] / out["lts"]["ms"]
    out["ideal_speedup"] = prob.n_el * n_fun / sum(int(c) * (n_fun >> g) for g, c in enumerate(counts))
    return out


def run_reference(a, ws, rank):
    """The reference arm: the reference's own vanilla CPU kernels (oracle/_ref) on the host cores,
    rank 0 only; each of the warm-up and timed steps is one step over the bounded sample of the
    workload (cpu_reference_rate). Nothing of the CUDA library is loaded on this path for elastic
    workloads."""
    if rank != 0:
        return
    w = WORKLOADS[a.workload]
    value, kind, cores, sample, extra = cpu_reference_rate(w.order, w.runs, w.rm, warm=a.warmup, steps=a.steps)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": a.workload, "reference_sample": sample},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample, **extra},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    a = parse()
    ws, rank, local = dist_init(a.gpus)
    if a.impl == "reference":
        run_reference(a, ws, rank)
        barrier(ws)
        return
    import numpy as np
    import torch
    from edge_b200 import _lib
    from edge_b200.solver import Solver

    torch.cuda.set_device(local)
    prob, prec = build_problem(a.workload)
    stream = torch.cuda.Stream()
    sv = Solver(prob, precision=prec, stream=stream.cuda_stream, device=local)
    e0, a0 = prob.zero_dofs(np.float32 if prec == 32 else np.float64)
    sv.upload_dofs(e0, a0)
    units_per_step = prob.n_el * prob.runs

    # warm-up, then K timed steps (inputs > L2: DOFs alone are several hundred MB)
    sv.step(a.warmup)
    sv.sync()
    clocks = Clocks(local)
    clocks.start()
    barrier(ws)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sv.step(a.steps)
    launches = sv.launches()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, ws)
    value = units_per_step * a.steps * ws / (ms_max / 1e3)

    # per-step latency and per-kernel times (a second pass with events around every launch)
    step_ms = []
    for _ in range(a.steps):
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        sv.step(1)
        e_b.record(stream)
        step_ms.append((e_a, e_b))
    torch.cuda.synchronize()
    step_ms = sorted(x.elapsed_time(y) for x, y in step_ms)
    L = _lib.lib()
    import ctypes as C
    L.edge_b200_set_timing(sv._h, 1)
    sv.step(a.steps)
    kms = np.zeros(4)
    kn = np.zeros(4, np.int64)
    L.edge_b200_kernel_times(sv._h, _lib.ptr(kms), _lib.ptr(kn))
    L.edge_b200_set_timing(sv._h, 0)
    names = ["local", "neighbour", "sources", "receivers"]
    shares = {names[i]: float(kms[i] / kms.sum()) for i in range(4) if kn[i]}
    kc = np.zeros(6, np.int32)
    L.edge_b200_kernel_config(sv._h, _lib.ptr(kc))
    alg = algorithmic(prob, prec, premix=bool(kc[1]), fs_pair=int(kc[2]), fused=bool(kc[5]), char=int(kc[1]) == 2)
    top = int(np.argmax(kms[:2]))
    avg_ms = kms[top] / max(kn[top], 1)
    # algorithmic bytes: the path's compulsory bytes of one element step (every array touched once:
    # DOFs read + written, time-integrated DOFs written + read once, FP64 star matrices and flux
    # solvers, connectivity) times the elements of the launch. The fused local kernel runs a whole
    # step per launch (this step's local update and the previous step's neighbour update); without
    # fusion the step's two kernels are timed together.
    fused = bool(kc[5])
    step_bytes = compulsory_step_bytes(prob, prec)
    bytes_launch = step_bytes * prob.n_el
    launch_ms = avg_ms if (fused and top == 0) else (kms[0] / max(kn[0], 1) + kms[1] / max(kn[1], 1))
    design_bytes = (alg["local_bytes"] if top == 0 else alg["neigh_bytes"]) * prob.n_el
    flops_launch = (alg["local_flops"] if top == 0 else alg["neigh_flops"]) * prob.n_el
    peak, peak_src = measured_peaks()
    achieved = bytes_launch / (launch_ms / 1e3) / 1e9
    traffic = traffic_from_profiles(a.workload)
    roofline = {"bound": "hbm", "kernel": names[top] if (fused and top == 0) else "local+neighbour",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_launch, "algorithmic_bytes_per_element_step": step_bytes,
                "launch_ms": launch_ms,
                "design_bytes_per_launch": design_bytes,
                "frac_design_bytes": design_bytes / (avg_ms / 1e3) / 1e9 / peak,
                "achieved_tflops": flops_launch / (avg_ms / 1e3) / 1e12,
                "kernel_avg_ms": {names[i]: float(kms[i] / kn[i]) for i in range(4) if kn[i]},
                "kernel_share": shares}
    # the local kernel is bound by the FP32 pipe, not HBM: its dense-equivalent flops (the DG
    # products counted dense; the kernel executes FMAs for the non-zeros only) against the nominal
    # FP32 CUDA-core peak (SMs x 128 FMA lanes x 2 flops x max SM clock)
    if prec == 32:
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        fp32_peak = sms * 128 * 2 * peak_clock_mhz() * 1e6 / 1e12
        roofline["fp32_pipe"] = {"dense_equivalent_tflops": roofline["achieved_tflops"],
                                 "nominal_peak_tflops": fp32_peak,
                                 "frac": roofline["achieved_tflops"] / fp32_peak}
    # the neighbour-flux kernel (the HBM-bound one) on its own: bytes this design moves (face
    # projections read, DOFs read + written, flux solvers, connectivity) and the reference algorithm's
    # count (neighbours' time-integrated DOFs instead of face projections)
    n_ms = kms[1] / max(kn[1], 1)
    B_, F_, p_ = host_n_modes(prob.order), prob.order * (prob.order + 1) // 2, (8 if prec == 64 else 4)
    ref_bytes = (3 * 9 * B_ * prob.runs * p_ + 4 * 81 * 8 + 4 * 6) * prob.n_el
    roofline_neighbour = {"bound": "hbm", "kernel": "neighbour", "avg_ms": n_ms,
                          "achieved": alg["neigh_bytes"] * prob.n_el / (n_ms / 1e3) / 1e9, "peak": peak,
                          "unit": "GB/s", "peak_source": peak_src,
                          "algorithmic_bytes_per_launch": alg["neigh_bytes"] * prob.n_el,
                          "achieved_reference_count": ref_bytes / (n_ms / 1e3) / 1e9}
    roofline_neighbour["frac"] = roofline_neighbour["achieved"] / peak
    roofline_neighbour["frac_reference_count"] = roofline_neighbour["achieved_reference_count"] / peak

    # end to end through the C ABI with host buffers: pinned H2D of the DOFs, one step, D2H of the DOFs
    pin_e = torch.from_numpy(e0).pin_memory()
    pin_a = torch.from_numpy(a0).pin_memory() if a0 is not None else None
    out_e = torch.empty_like(pin_e).pin_memory()
    out_a = torch.empty_like(pin_a).pin_memory() if pin_a is not None else None
    ke = a.e2e_steps
    barrier(ws)
    torch.cuda.synchronize()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    L.edge_b200_join_transfers(sv._h, 1)
    for _ in range(ke):
        # copies in both directions on the context's copy streams, overlapping each other and the step
        L.edge_b200_upload_dofs_async(sv._h, C.c_void_p(pin_e.data_ptr()),
                                      C.c_void_p(pin_a.data_ptr()) if pin_a is not None else None)
        sv.step(1)
        L.edge_b200_download_dofs_async(sv._h, C.c_void_p(out_e.data_ptr()),
                                        C.c_void_p(out_a.data_ptr()) if out_a is not None else None)
    L.edge_b200_join_transfers(sv._h, 0)
    x1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(x0.elapsed_time(x1), ws)
    dof_bytes = pin_e.numel() * pin_e.element_size() + (pin_a.numel() * pin_a.element_size() if pin_a is not None else 0)
    # the copies' own bound on this host: 1 GiB each way at once between the same pinned buffers
    # and the device (CUDA events on two streams), after the timed region
    nb = min(1 << 30, pin_e.numel() * pin_e.element_size())
    hb = pin_e.view(-1).view(torch.uint8)[:nb]
    ob = out_e.view(-1).view(torch.uint8)[:nb]
    dev_a = torch.empty(nb, dtype=torch.uint8, device=local)
    dev_b = torch.empty(nb, dtype=torch.uint8, device=local)
    s_up, s_dn = torch.cuda.Stream(device=local), torch.cuda.Stream(device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for rep in range(2):  # the first pass warms the copy engines
        torch.cuda.synchronize()
        ev[0].record(s_up)
        ev[2].record(s_dn)
        with torch.cuda.stream(s_up):
            dev_a.copy_(hb, non_blocking=True)
        with torch.cuda.stream(s_dn):
            ob.copy_(dev_b, non_blocking=True)
        ev[1].record(s_up)
        ev[3].record(s_dn)
        torch.cuda.synchronize()
    h2d_gbs = nb / (ev[0].elapsed_time(ev[1]) / 1e3) / 1e9
    d2h_gbs = nb / (ev[2].elapsed_time(ev[3]) / 1e3) / 1e9
    del dev_a, dev_b
    bound_s = max(dof_bytes / (h2d_gbs * 1e9), dof_bytes / (d2h_gbs * 1e9))
    e2e = {"value": units_per_step * ke * ws / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": dof_bytes,
           "d2h_bytes_per_step": dof_bytes, "steps": ke,
           "pcie_gbs_both_directions_at_once": {"h2d": h2d_gbs, "d2h": d2h_gbs},
           "copy_bound_value": units_per_step / bound_s,
           "frac_of_copy_bound": (units_per_step * ke / (e2e_ms / 1e3)) / (units_per_step / bound_s),
           "note": "per step: pinned host->device DOFs, one GTS step, device->host DOFs (the drop-in for "
                   "host-resident DOFs), asynchronous copies overlapping across steps; copy_bound_value: the "
                   "rate if each step took only its DOFs' copies at the measured bandwidth"}

    # plain FP64 path on the same mesh (one run) for the batched-FP32 vs plain-FP64 ratio
    fp64 = None
    if not a.no_fp64 and prec == 32 and prob.rm == 0:
        from edge_b200 import host
        p64 = host.Problem(order=prob.order, runs=1, rm=0, mesh=prob.mesh, rho=prob.rho, lam=prob.lam,
                           mu=prob.mu, starE=prob.starE, fsE=prob.fsE, dt=prob.dt, name="fp64")
        s64 = Solver(p64, precision=64, stream=stream.cuda_stream, device=local)
        z, _ = p64.zero_dofs()
        s64.upload_dofs(z)
        s64.step(2)
        s64.sync()
        k64 = max(20, a.steps)
        y0, y1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        y0.record(stream)
        s64.step(k64)
        y1.record(stream)
        torch.cuda.synchronize()
        v64 = prob.n_el * k64 / (y0.elapsed_time(y1) / 1e3)
        fp64 = {"value": v64 * ws, "unit": UNIT, "ms_per_step": y0.elapsed_time(y1) / k64,
                "config": {"order": prob.order, "runs": 1, "precision": "fp64"},
                "batched_fp32_over_plain_fp64": value / (v64 * ws)}
        # the plain path against both ceilings: HBM (its algorithmic bytes per element) and the FP64
        # pipe (dense-equivalent flops over the nominal SMs x 64 FP64 FMA lanes x 2 x max SM clock)
        alg64 = algorithmic(p64, 64)
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        fp64_peak = sms * 64 * 2 * peak_clock_mhz() * 1e6 / 1e12
        tfl = (alg64["local_flops"] + alg64["neigh_flops"]) * v64 / 1e12
        gbs = (alg64["local_bytes"] + alg64["neigh_bytes"]) * v64 / 1e9
        fp64["fp64_pipe"] = {"dense_equivalent_tflops": tfl, "nominal_peak_tflops": fp64_peak, "frac": tfl / fp64_peak}
        fp64["hbm"] = {"achieved_gbs": gbs, "peak": peak, "frac": gbs / peak, "peak_source": peak_src}
        s64.close()

    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        v, kind, cores, sample, extra = cpu_reference_rate(prob.order, prob.runs, prob.rm)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample, **extra}

    sv.close()
    # the FP32 error bar at the workload's full size and stated step count: per fused run, the
    # receivers against the same run alone on the plain FP64 path (pinned to the oracle to 1e-12)
    parity = None
    if a.parity and rank == 0 and prec == 32:
        from edge_b200 import accuracy
        parity = accuracy.fused_vs_plain(prob, WORKLOADS[a.workload].steps, device=local)
        parity["tolerance"] = 1e-4
        parity["within_tolerance"] = parity["receiver_rel_l2_max"] < 1e-4
    tc = None
    if a.tc_probe and rank == 0:
        try:
            tc = run_tc_probe(roofline["kernel_avg_ms"]["local"], prob.n_el, prob.order, prob.runs, local,
                              clk["sm_mhz"] or peak_clock_mhz())
        except (RuntimeError, OSError) as e:
            tc = {"unavailable": str(e)}
    serving = None
    if a.serve_requests > 0:
        serving = run_serve(a.serve_requests, a.serve_rate, local)
    lts = run_lts(local) if a.lts_report else None
    batch = run_batch(a.batch_sims, local) if (a.batch_sims > 0 and rank == 0) else None

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == 32 else "f64",
               "data": "synthetic",
               "config": {"workload": a.workload, "tets": prob.n_el, "order": prob.order, "runs": prob.runs,
                          "mechanisms": prob.rm, "precision": f"fp{prec}", "parallelism": f"replicas{ws}",
                          "l2": "inputs larger than L2 (DOFs %.0f MB)" % (dof_bytes / 1e6),
                          "dt": prob.dt},
               "step_ms_p50": step_ms[len(step_ms) // 2], "step_ms_p99": step_ms[min(len(step_ms) - 1,
                                                                                      int(0.99 * len(step_ms)))],
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
               "clocks": clk, "fp64_plain": fp64, "serving": serving, "roofline_neighbour": roofline_neighbour, "lts": lts,
               "batch": batch, "parity_at_size": parity, "tensor_core_probe": tc}
        print(json.dumps(out), flush=True)
    barrier(ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
