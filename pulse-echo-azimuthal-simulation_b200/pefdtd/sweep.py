"""Resumable azimuth sweeps, batched on one GPU.

Same sweep definition, files and control protocol as the reference's
sweep engine (sim/pipeline/sweep_runner.py), so its tools can read and
continue these sweeps:

  <root>/<name>/config.json    the sweep definition (DEFAULTS + overrides,
                               written once)
  <root>/<name>/az{ddd}.npz    one file per completed azimuth, written to a
                               ``.tmp.npz`` name and renamed into place:
                               trace (f32), dt, f0, az_deg, E1, t1_s,
                               coda_db, tail, h, order, ppw, fluid_damp, seed
  <root>/<name>/status.json    merge-updated heartbeat (pid, heartbeat,
                               done, total, phase, current_az, sec_per_az)
  <root>/<name>/STOP           cooperative stop: checked before each batch
                               and between graph chunks; in-flight azimuths
                               are dropped and redone on continue

Per azimuth (sweep_runner.py:322-390): the specimen and its c-axes rotated
by -az against the fixed probe (single-raster Laguerre evaluation, or the
legacy nearest resample), ice tables, dt = safe_dt_labels(safety 0.5),
nt = record_factor * D / C_REF / dt, a Ricker wavelet at f0, fluid damping
exp(-fluid_damp * EDT) outside the ice, and a piston of element_d_mm on the
+x rim, recorded as mean pressure; then analyse_trace's (E1, t1, coda, tail).

Different from the reference: instead of one solve per azimuth, ``batch``
pending azimuths (default: as many as fit in device memory) run as one
:class:`pefdtd.batch.BatchSolver`, each solve bit-identical to its own
``forward_fused_labels`` call (shorter records are zero-padded to the
longest and cut back), while the next batch's grids, tables and masks are
prepared on host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import coeffs as _coeffs
from . import damping, materials, specimen, wavelets

C_REF = 3850.0

DEFAULTS = dict(
    f0_mhz=5.0, ppw=6.0, order=8, az_start=0, az_stop=360, az_step=1,
    sweep_order="progressive", record_factor=2.7, fluid_damp=0.02, sponge=10,
    element_d_mm=6.35, diameter_mm=100.0, thickness_mm=35.0, n_grains=100,
    size_cv=0.35, concentration=3.93, spatial_corr=0.0, fabric_axis=[1.0, 0.0, 0.0],
    seed=7, axes_convention="rigid2", fd_kh_max=2.0, rasterise="single",
)


class StopRequested(Exception):
    pass


# ---------------------------------------------------------------- files
def sweeps_root(root=None):
    if root is not None:
        return root
    return os.environ.get("PEFDTD_SWEEPS", os.path.join(os.getcwd(), "out", "sweeps"))


def sweep_dir(name, root=None):
    return os.path.join(sweeps_root(root), name)


def _replace(tmp, dst, critical):
    """os.replace, retried while another process briefly holds the target
    (a reader polling status.json); data files must land, status may not."""
    for _ in range(25):
        try:
            os.replace(tmp, dst)
            return True
        except PermissionError:
            time.sleep(0.2)
    if critical:
        raise PermissionError(f"could not replace {dst}: something keeps it open")
    try:
        os.remove(tmp)
    except OSError:
        pass
    return False


def create(name, root=None, **overrides):
    cfg = dict(DEFAULTS)
    cfg.update(overrides)
    cfg["name"] = name
    d = sweep_dir(name, root)
    os.makedirs(d, exist_ok=True)
    p = os.path.join(d, "config.json")
    if not os.path.exists(p):
        with open(p, "w", encoding="utf-8") as f:
            json.dump(cfg, f, indent=1)
    return p


def load(name_or_path, root=None):
    p = (name_or_path if name_or_path.endswith("config.json")
         else os.path.join(sweep_dir(name_or_path, root), "config.json"))
    with open(p, encoding="utf-8") as f:
        cfg = json.load(f)
    cfg.setdefault("_root", os.path.dirname(os.path.dirname(os.path.abspath(p))))
    return cfg


def list_sweeps(root=None):
    r = sweeps_root(root)
    if not os.path.isdir(r):
        return []
    return [n for n in sorted(os.listdir(r)) if os.path.exists(os.path.join(r, n, "config.json"))]


def _root_of(cfg, root):
    return root if root is not None else cfg.get("_root")


# ---------------------------------------------------------------- order
def bit_reversed_order(n):
    """Van der Corput order of range(n): each index i of the next power of
    two 2^b is visited as reverse_bits_b(i), skipping values >= n, so every
    prefix is spread near-uniformly over the range."""
    if n <= 1:
        return list(range(n))
    b = (n - 1).bit_length()
    i = np.arange(1 << b)
    r = np.zeros_like(i)
    for k in range(b):
        r |= ((i >> k) & 1) << (b - 1 - k)
    return [int(v) for v in r if v < n]


def azimuths(cfg):
    """Visiting order: 'progressive' takes the first half-circle
    [az_start, az_start + 180) in bit-reversed order, then the rest the same
    way (the fabric observables repeat every 180 degrees); otherwise plain
    order."""
    base = list(range(int(cfg["az_start"]), int(cfg["az_stop"]), int(cfg["az_step"])))
    if cfg.get("sweep_order", "progressive") != "progressive":
        return base
    mid = cfg["az_start"] + 180
    first = [a for a in base if a < mid]
    second = [a for a in base if a >= mid]
    return [first[i] for i in bit_reversed_order(len(first))] + \
           [second[i] for i in bit_reversed_order(len(second))]


def done_azimuths(cfg, root=None):
    d = sweep_dir(cfg["name"], _root_of(cfg, root))
    return sorted(int(f[2:5]) for f in os.listdir(d)
                  if f.startswith("az") and f.endswith(".npz") and not f.endswith(".tmp.npz"))


def pending(cfg, root=None):
    done = set(done_azimuths(cfg, root))
    return [a for a in azimuths(cfg) if a not in done]


_status_lock = threading.Lock()


def status(cfg, root=None, **kw):
    """Merge-update status.json: fields known only while running
    (sec_per_az) survive a later write that does not carry them."""
    root = _root_of(cfg, root)
    p = os.path.join(sweep_dir(cfg["name"], root), "status.json")
    with _status_lock:
        s = {}
        if os.path.exists(p):
            try:
                with open(p, encoding="utf-8") as f:
                    s = json.load(f)
            except Exception:
                s = {}
        s.update(pid=os.getpid(), heartbeat=time.time(), done=len(done_azimuths(cfg, root)),
                 total=len(azimuths(cfg)))
        s.update({k: v for k, v in kw.items() if v is not None})
        tmp = p + ".tmp"
        with open(tmp, "w", encoding="utf-8") as f:
            json.dump(s, f)
        _replace(tmp, p, critical=False)


def analyse(tr, dt):
    """(E1, t1_s, coda_db, tail) of one trace: first echo on the 2 x 100 mm
    round trip (sweep_runner.py:206-222)."""
    return wavelets.analyse_trace(tr, dt, path_m=0.200, c_ref=C_REF)


def save_azimuth(cfg, az, tr, dt, f0, h, root=None, analysis=None):
    """Write az{ddd}.npz; ``analysis`` = (E1, t1, coda, tail) computed
    elsewhere (the device batch analysis), else computed here on the host."""
    d = sweep_dir(cfg["name"], _root_of(cfg, root))
    tr = np.asarray(tr, float).ravel()
    E1, t1, coda, tail = analyse(tr, dt) if analysis is None else analysis
    tmp = os.path.join(d, f"az{az:03d}.tmp.npz")
    np.savez(tmp, trace=tr.astype(np.float32), dt=dt, f0=f0, az_deg=az, E1=E1, t1_s=t1,
             coda_db=coda, tail=tail, h=h, order=cfg["order"], ppw=cfg["ppw"],
             fluid_damp=cfg["fluid_damp"], seed=cfg["seed"])
    _replace(tmp, os.path.join(d, f"az{az:03d}.npz"), critical=True)
    return E1, t1, coda, tail


# ---------------------------------------------------------------- per azimuth
def sweep_coeffs(cfg):
    """FD coefficients: the multistart kh_max solve, or the single-start
    kh_max 1.6 set for configs written before fd_kh_max existed."""
    khm = cfg.get("fd_kh_max")
    return _coeffs.optimised_coeffs(cfg["order"], kh_max=1.6 if khm is None else float(khm),
                                    multistart=khm is not None)


def rim_piston(lab, nd, element_d_mm, h):
    """Piston cells on the +x rim: the last ice column of the centre row
    (one cell inside the rim), a disc of radius element_d/2 in (y, z),
    fluid cells dropped; (dy, dz) row-major order as the reference lists
    them (sweep_runner.py:342-351)."""
    nz, ny = lab.shape[0], lab.shape[1]
    cz, cy, cx = nz // 2, ny // 2, ny // 2
    Rc = nd // 2
    ks = np.arange(Rc - 1, 0, -1)
    hit = ks[lab[cz, cy, cx + ks] >= 0]
    if len(hit) == 0:
        raise ValueError("no ice on the +x radius of the centre plane")
    ixp = cx + int(hit[0]) - 1
    er = max(int(element_d_mm * 1e-3 / 2 / h), 1)
    pts = [(cz + dz, cy + dy, ixp) for dy in range(-er, er + 1) for dz in range(-er, er + 1)
           if dy * dy + dz * dz <= er * er and lab[cz + dz, cy + dy, ixp] >= 0]
    return pts


def azimuth_setup(cfg, build, co, az, labeller=None):
    """Solve description (pefdtd.fdtd.label_solve_spec) of one azimuth plus
    its dt, nt, f0, h."""
    from .fdtd import label_solve_spec
    f0 = cfg["f0_mhz"] * 1e6
    h = C_REF / f0 / cfg["ppw"]
    if cfg.get("rasterise") == "single":
        lab, nd, _, axes_rot = specimen.rotated_grid_single_raster(build, h, cfg["sponge"], az,
                                                                   labeller=labeller)
    elif specimen.pick_labeller(labeller=labeller) == "gpu":
        # the same resample on the device (bit-identical), read back for the
        # host-side probe, damping mask and time step
        lab_d, nd, _, axes_rot = specimen.rotated_grid_device(build["labels"], build["axes"], build["h"],
                                                              h, cfg["sponge"], az)
        lab = lab_d.cpu().numpy()
    else:
        lab, nd, _, axes_rot = specimen.rotated_grid(build["labels"], build["axes"], build["h"], h,
                                                     cfg["sponge"], az)
    Ct, rho_t = materials.material_tables(axes_rot)
    # material indices as uint8, as the reference computes this dt (it wraps
    # above 254 grains; kept so that dt, nt and the files stay identical)
    dt = damping.safe_dt_labels((lab + 1).astype(np.uint8), Ct, rho_t, h, co, 0.5)
    nt = int(cfg["record_factor"] * nd * h / C_REF / dt)
    wav = wavelets.ricker(f0, dt, nt)
    dm = damping.fluid_damp_mask(lab, cfg["fluid_damp"])
    pts = rim_piston(lab, nd, cfg["element_d_mm"], h)
    w = 1.0 / len(pts)
    spec = label_solve_spec(lab, axes_rot, h, dt, nt, [(p, w) for p in pts], wav,
                            [(pts, np.full(len(pts), w))], order=cfg["order"], coeffs=co,
                            sponge_width=cfg["sponge"], damp_mask=dm, mat_tables=(Ct, rho_t))
    return dict(az=az, spec=spec, dt=dt, nt=nt, f0=f0, h=h, axes=axes_rot)


def setup_bytes(setup, dtype_size=4):
    """Device bytes one solve of this setup holds: nine fields, labels,
    damping volume, traces."""
    cells = int(np.prod(setup["spec"]["mats"].shape))
    return cells * (9 * dtype_size + 2 + 4) + setup["nt"] * dtype_size + (64 << 20)


# ---------------------------------------------------------------- solving
def solve_batch(setups, progress=None, device=None, chunk_steps=200):
    """Traces (nt_i,) of several azimuth setups run as one GPU batch; every
    record is zero-padded to the longest and cut back, so each equals its
    own forward_fused_labels call. ``progress(frac)`` runs between chunks
    and may raise to abandon the batch."""
    from .batch import BatchSolver
    nt_max = max(s["nt"] for s in setups)
    specs = []
    for s in setups:
        sp = dict(s["spec"])
        w = np.zeros(nt_max)
        w[:s["nt"]] = sp["wavelet"][:s["nt"]]
        sp["wavelet"] = w
        specs.append(sp)
    b = BatchSolver(specs, device=device, chunk_steps=chunk_steps)
    try:
        n = 0
        while n < nt_max:
            m = min(nt_max, n + chunk_steps)
            b.run(n, m)
            n = m
            if progress is not None:
                b.torch.cuda.current_stream(b.device).synchronize()
                progress(n / nt_max)
        out = b.traces_numpy(nt_max)
    finally:
        b.close()
    return [np.asarray(tr[:s["nt"], 0], float) for tr, s in zip(out, setups)]


def _device_budget(device=None):
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    return int(free * 0.85)


def run(cfg, root=None, batch=None, device=None, labeller=None, log=print, solver=None,
        prefetch=True, rank=0, world=1):
    """Run (or continue) a sweep. ``batch``: azimuths per GPU batch (None =
    as many as fit in device memory). ``labeller``: see
    specimen.DiskSpecimen.build. ``solver``: callable(setups, progress) ->
    traces; the GPU batch solver unless replaced (tests drive the file
    protocol on CPU with a stand-in). With the GPU solver each batch's
    figures (E1, t1, coda, tail) are computed on the device
    (:func:`pefdtd.traces.analyse`: t1 identical to the host analysis, the
    others to ~1e-13 relative); with a stand-in, on the host, exactly as the
    reference computes them. ``rank``/``world``: one process per
    GPU, in an initialised torch.distributed process group; each rank solves
    its share (:func:`pefdtd.shard.assign`, every azimuth of a sweep costs
    the same) of rank 0's list of pending azimuths, broadcast to all, and
    writes their files; rank 0 alone writes status.json and config.json."""
    root = _root_of(cfg, root)
    if world > 1 and rank != 0:
        status = lambda *a, **k: None  # noqa: E731,F841  (rank 0 owns status.json)
    else:
        status = globals()["status"]
    device_analysis = solver is None
    if solver is None:
        try:
            import torch
            ok = torch.cuda.is_available()
        except Exception:
            ok = False
        if not ok:
            status(cfg, root, phase="NO CUDA - cannot run")
            log("[sweep] CUDA unavailable: the full-wave solver needs an NVIDIA GPU.")
            return "no-cuda"
        solver = lambda setups, progress: solve_batch(setups, progress, device=device)  # noqa: E731
    d = sweep_dir(cfg["name"], root)
    stop_flag = os.path.join(d, "STOP")
    # shared files change on rank 0 alone (a stale STOP flag, config.json);
    # the other ranks reach their first read of them after the pending-list
    # broadcast below, which rank 0 joins only after these writes
    if rank == 0 and os.path.exists(stop_flag):
        os.remove(stop_flag)
    if cfg.get("axes_convention") != "rigid2":
        if done_azimuths(cfg, root):
            status(cfg, root, phase="LEGACY sweep - cannot continue")
            log("[sweep] config has no axes_convention='rigid2' and finished azimuths: the "
                "rigid-rotation convention would mix with the old one. Start a new sweep.")
            return "legacy"
        cfg["axes_convention"] = "rigid2"
        if rank == 0:
            p = os.path.join(d, "config.json")
            tmp = p + ".tmp"
            keep = {k: v for k, v in cfg.items() if not k.startswith("_")}
            with open(tmp, "w", encoding="utf-8") as f:
                json.dump(keep, f, indent=1)
            _replace(tmp, p, critical=True)

    f0 = cfg["f0_mhz"] * 1e6
    h = C_REF / f0 / cfg["ppw"]
    log(f"[sweep {cfg['name']}] building specimen (h = {h * 1e3:.3f} mm)")
    hb_stop = threading.Event()

    def _hb():
        while not hb_stop.is_set():
            status(cfg, root, phase=f"building specimen (h = {h * 1e3:.2f} mm)")
            hb_stop.wait(20)
    threading.Thread(target=_hb, daemon=True).start()
    try:
        sp = specimen.DiskSpecimen(diameter_m=cfg["diameter_mm"] * 1e-3,
                                   thickness_m=cfg["thickness_mm"] * 1e-3, n_grains=cfg["n_grains"],
                                   size_cv=cfg["size_cv"], concentration=cfg["concentration"],
                                   spatial_corr=cfg["spatial_corr"],
                                   fabric_axis=tuple(cfg["fabric_axis"]), seed=cfg["seed"])
        build = sp.build(h, labeller=labeller)
    finally:
        hb_stop.set()
    co = sweep_coeffs(cfg)
    todo = pending(cfg, root)
    if world > 1:
        # every rank shards rank 0's list: a rank that read the directory
        # after another had written files would see a shorter one, and the
        # shares would no longer cover the pending azimuths
        import torch.distributed as dist
        from .shard import assign
        box = [todo]
        dist.broadcast_object_list(box, src=0)
        todo = box[0]
        todo = [todo[i] for i in assign([1.0] * len(todo), world)[rank]]
    log(f"[sweep] {len(todo)} of {len(azimuths(cfg))} azimuths pending"
        + (f" on rank {rank} of {world}" if world > 1 else ""))
    if not todo:
        status(cfg, root, phase="complete")
        return "complete"

    setup = lambda az: azimuth_setup(cfg, build, co, az, labeller=labeller)  # noqa: E731
    first = setup(todo[0])
    if batch is None:
        per = setup_bytes(first)
        try:
            batch = max(1, _device_budget(device) // per)
        except Exception:
            batch = 1
    batch = max(1, min(int(batch), len(todo)))
    groups = [todo[i:i + batch] for i in range(0, len(todo), batch)]
    pool = ThreadPoolExecutor(max_workers=min(8, batch)) if prefetch else None

    def prepare(group, have=None):
        have = have or {}
        if pool is None:
            return [have.get(a) or setup(a) for a in group]
        futs = [None if a in have else pool.submit(setup, a) for a in group]
        return [have[a] if f is None else f.result() for a, f in zip(group, futs)]

    def prepare_async(group):
        if pool is None:
            return None
        return [pool.submit(setup, a) for a in group]

    times = []
    result = "complete"
    try:
        cur = prepare(groups[0], {todo[0]: first})
        nxt_f = prepare_async(groups[1]) if len(groups) > 1 else None
        for gi, group in enumerate(groups):
            if os.path.exists(stop_flag):
                log("[sweep] STOP flag found - exiting; completed azimuths are saved.")
                status(cfg, root, phase="stopped")
                result = "stopped"
                break
            t0 = time.time()
            label = f"az {group[0]}" if len(group) == 1 else f"az {group[0]}..{group[-1]} ({len(group)})"
            spa = float(np.mean(times)) if times else None
            status(cfg, root, phase=label, current_az=group[0], sec_per_az=spa)

            def prog(frac, label=label, group=group, spa=spa):
                status(cfg, root, phase=f"{label} ({100 * frac:.0f}%)", current_az=group[0],
                       sec_per_az=spa)
                if os.path.exists(stop_flag):
                    raise StopRequested()
            try:
                traces = solver(cur, prog)
            except StopRequested:
                log(f"[sweep] STOP mid-batch at {label}: these azimuths are redone on continue.")
                status(cfg, root, phase="stopped")
                result = "stopped"
                break
            if device_analysis:
                # the batch's E1 / arrival / coda / tail in one device pass
                from . import traces as trace_ops
                figs = trace_ops.analyse(traces, [s["dt"] for s in cur], path_m=0.200, c_ref=C_REF,
                                         device=device)
            else:
                figs = [None] * len(cur)
            for s, tr, fig in zip(cur, traces, figs):
                E1, t1, coda, tail = save_azimuth(cfg, s["az"], tr, s["dt"], s["f0"], s["h"], root,
                                                  analysis=fig)
                log(f"[sweep] az {s['az']:3d}: coda {coda:6.1f} dB, E1 {E1:.4g}, "
                    f"ToF {t1 * 1e6:.3f} us, tail {tail:.3f} "
                    f"({'STABLE' if tail < 0.5 else 'CHECK'})")
            el = (time.time() - t0) / len(group)
            times.extend([el] * len(group))
            if gi + 1 < len(groups):
                cur = [f.result() for f in nxt_f] if nxt_f is not None else prepare(groups[gi + 1])
                nxt_f = prepare_async(groups[gi + 2]) if gi + 2 < len(groups) else None
    finally:
        if pool is not None:
            pool.shutdown(wait=True, cancel_futures=True)
    if result == "complete":
        status(cfg, root, phase="complete", sec_per_az=float(np.mean(times)) if times else None)
        log("[sweep] COMPLETE")
    return result


def main(argv=None):
    ap = argparse.ArgumentParser(description="resumable batched azimuth sweeps")
    ap.add_argument("--run", help="sweep name or config.json path")
    ap.add_argument("--new", help="create a sweep with this name")
    ap.add_argument("--set", nargs="*", default=[], help="key=value overrides for --new")
    ap.add_argument("--root", default=None, help="sweeps directory (default $PEFDTD_SWEEPS or ./out/sweeps)")
    ap.add_argument("--batch", type=int, default=None, help="azimuths per GPU batch")
    a = ap.parse_args(argv)
    if a.new:
        kw = {}
        for kv in a.set:
            k, v = kv.split("=", 1)
            try:
                kw[k] = json.loads(v)
            except json.JSONDecodeError:
                kw[k] = v
        print(f"created {create(a.new, a.root, **kw)}")
        return
    if a.run:
        run(load(a.run, a.root), a.root, batch=a.batch)


if __name__ == "__main__":
    main()
