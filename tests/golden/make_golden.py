"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container that holds the reference sources, built into oracle/_ref first
(their path: REF=<dir> or the CABLEGEN_REFERENCE environment variable):

    make -C oracle all REF=<reference sources> # builds oracle/_ref/{libcgref.so,cli}
    python tests/golden/make_golden.py units
    python tests/golden/make_golden.py run plain_2x4 --cores 8
    python tests/golden/make_golden.py run ll_unpruned --end 120 --cores 8
    python tests/golden/make_golden.py run ll_pruned --cores 8   # full size, long

`units` writes known-answer vectors for the board primitives by calling the
reference library's own functions (canonicalize_b, movedir_unstable,
prune_board, the row LUT, lookup, cmpbrd, expectimax).  `run` drives the
reference CLI (`cli -C=conf -c=N generate` then `solve`) on a seeded workload
and records, per layer, the board count and the SHA-256 of the reference's
`.boards` file and `.tables` file, plus (for small layers) the raw files.

The GPU box has no reference; it only reads the JSON/binary fixtures.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from cablegen_b200 import configs  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libcgref.so")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "cli")


def write_conf(path, wl: configs.Workload, form: configs.Formation, bdir, tdir, cores, end_gen=None,
               end_solve=None):
    configs.reference_conf(path, wl, form, bdir, tdir, cores, end_gen=end_gen, end_solve=end_solve)


def sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        while True:
            b = f.read(1 << 24)
            if not b:
                break
            h.update(b)
    return h.hexdigest()


def prepare(name, end, work, cores):
    wl = configs.get(name) if end is None else configs.get(name, end_gen=end)
    form = wl.formations[0]
    os.makedirs(work, exist_ok=True)
    bdir = os.path.join(work, "boards") + "/"
    tdir = os.path.join(work, "tables") + "/"
    os.makedirs(bdir, exist_ok=True)
    os.makedirs(tdir, exist_ok=True)
    np.array(form.initial, dtype="<u8").tofile(os.path.join(work, "initial"))
    np.array(form.winstates, dtype="<u8").tofile(os.path.join(work, "winstates"))
    conf = os.path.join(work, "cablegen.conf")
    write_conf(conf, wl, form, bdir, tdir, cores)
    return wl, form, conf, bdir, tdir


def hash_tables_streaming(tdir, form, proc, rec):
    """Hash each .tables file once the solver has moved past it, then delete it.

    The reference solves top-down and writes <s>.tables at the end of layer s;
    when <s-2>.tables appears (or the solver exits) layer s is complete.  Large
    workloads do not fit on disk otherwise.
    """
    sums = list(range(form.end_gen, form.start - 1, -2))
    i = 0
    while i < len(sums):
        s = sums[i]
        p = os.path.join(tdir, f"{s}.tables")
        nxt = os.path.join(tdir, f"{s - 2}.tables") if i + 1 < len(sums) else None
        done = proc.poll() is not None
        if os.path.exists(p) and (done or (nxt and os.path.exists(nxt))):
            n = rec[str(s)]["boards"]
            rec[str(s)]["tables_sha256"] = sha(p)
            vals = np.fromfile(p, dtype="<f8")[n:]
            rec[str(s)]["max_p"] = float(vals.max()) if len(vals) else 0.0
            rec[str(s)]["sum_p"] = float(vals.sum()) if len(vals) else 0.0
            os.remove(p)
            i += 1
            continue
        if done and not os.path.exists(p):
            raise RuntimeError(f"solver exited without writing {p}")
        time.sleep(0.05)


def run_workload(name, cores, end=None, keep_dir=None, solve=True, reuse=False):
    work = keep_dir or tempfile.mkdtemp(prefix=f"golden_{name}_")
    wl, form, conf, bdir, tdir = prepare(name, end, work, cores)
    out = {"workload": name, "description": wl.description, "start": form.start,
           "end_gen": form.end_gen, "cores": cores, "layers": {}}
    if not (reuse and os.path.exists(os.path.join(bdir, f"{form.end_gen}.boards"))):
        t0 = time.time()
        subprocess.run([REF_CLI, f"-C={conf}", f"-c={cores}", "generate"], check=True, cwd=work,
                       stdout=subprocess.DEVNULL)
        out["gen_seconds"] = round(time.time() - t0, 2)
    for s in range(form.start, form.end_gen + 1, 2):
        p = os.path.join(bdir, f"{s}.boards")
        n = os.path.getsize(p) // 8
        out["layers"][str(s)] = {"boards": n, "boards_sha256": sha(p)}
    if solve:
        t0 = time.time()
        proc = subprocess.Popen([REF_CLI, f"-C={conf}", f"-c={cores}", "solve"], cwd=work,
                                stdout=subprocess.DEVNULL)
        hash_tables_streaming(tdir, form, proc, out["layers"])
        if proc.wait() != 0:
            raise RuntimeError("reference solve failed")
        out["solve_seconds"] = round(time.time() - t0, 2)
    return out, work, bdir, tdir


def cmd_run(args):
    out, work, bdir, tdir = run_workload(args.workload, args.cores, args.end, args.keep, not args.no_solve,
                                         args.reuse)
    tag = args.workload if args.end is None else f"{args.workload}_end{args.end}"
    store = os.path.join(HERE, tag)
    os.makedirs(store, exist_ok=True)
    with open(os.path.join(store, "digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps({k: v for k, v in out.items() if k != "layers"}), "layers:", len(out["layers"]),
          "total boards:", sum(r["boards"] for r in out["layers"].values()))
    if not args.keep:
        shutil.rmtree(work)


# ---------------------------------------------------------------- CLI transcripts
CLI_WORKLOAD = "plain_2x4_nearwall"
CLI_LOOKUPS = ["0x33301231ffffffff", "0x12000000ffffffff", "0x1123331ffffffff", "0x30100021ffffffff"]
CLI_SPAWN_LOOKUPS = ["0x33311231ffffffff"]


def cli_prepare(work, cores=2):
    """Config with relative paths, so transcripts do not depend on the directory."""
    wl = configs.get(CLI_WORKLOAD)
    form = wl.formations[0]
    os.makedirs(os.path.join(work, "boards"), exist_ok=True)
    os.makedirs(os.path.join(work, "tables"), exist_ok=True)
    np.array(form.initial, dtype="<u8").tofile(os.path.join(work, "initial"))
    np.array(form.winstates, dtype="<u8").tofile(os.path.join(work, "winstates"))
    conf = os.path.join(work, "cablegen.conf")
    write_conf(conf, wl, form, "./boards/", "./tables/", cores)
    with open(conf) as f:
        text = f.read()
    text = text.replace(os.path.join(work, "initial"), "./initial").replace(os.path.join(work, "winstates"), "./winstates")
    with open(conf, "w") as f:
        f.write(text)
    return "cablegen.conf"


def cli_commands():
    cmds = [["lookup", b] for b in CLI_LOOKUPS] + [["lookup_spawn", b] for b in CLI_SPAWN_LOOKUPS]
    cmds += [["explore", "./tables/16.tables"], ["read", "./boards/14.boards"]]
    return cmds


# play and train draw spawns from rand() seeded with time(NULL) (frontends/cli/main.c:354-475);
# with time() fixed by a preloaded library both CLIs replay the same game.  train reads
# its moves from standard input.
CLI_GAMES = [("play", "0x12000000ffffffff", ""), ("train", "0x12000000ffffffff", "asdwdsaw" * 40)]


def fixed_time_lib(outdir):
    """Builds tests/host/fixed_time.c into outdir/fixed_time.so (gcc) and returns its path."""
    out = os.path.join(outdir, "fixed_time.so")
    src = os.path.join(HERE, "..", "host", "fixed_time.c")
    subprocess.run(["gcc", "-shared", "-fPIC", "-O2", "-o", out, src], check=True)
    return out


def run_game(cli, conf, work, env, cmd, board, stdin, preload):
    env = dict(env, LD_PRELOAD=preload)
    r = subprocess.run([cli, f"-C={conf}", cmd, board], cwd=work, env=env, input=stdin, capture_output=True,
                       text=True, timeout=300)
    return r.stdout


def cmd_cli(args):
    work = tempfile.mkdtemp(prefix="golden_cli_")
    conf = cli_prepare(work)
    env = dict(os.environ, XDG_CONFIG_HOME=work)
    for c in ("generate", "solve"):
        subprocess.run([REF_CLI, f"-C={conf}", c], check=True, cwd=work, env=env, stdout=subprocess.DEVNULL)
    store = os.path.join(HERE, "cli")
    os.makedirs(store, exist_ok=True)
    for i, c in enumerate(cli_commands()):
        out = subprocess.run([REF_CLI, f"-C={conf}"] + c, cwd=work, env=env, capture_output=True, text=True).stdout
        with open(os.path.join(store, f"{i:02d}_{c[0]}.txt"), "w") as f:
            f.write(out)
    preload = fixed_time_lib(work)
    for cmd, board, stdin in CLI_GAMES:
        out = run_game(REF_CLI, conf, work, env, cmd, board, stdin, preload)
        with open(os.path.join(store, f"game_{cmd}.txt"), "w") as f:
            f.write(out)
    shutil.rmtree(work)
    print("cli transcripts:", len(cli_commands()), "games:", len(CLI_GAMES))


# ---------------------------------------------------------------- unit vectors
class MinSettings(C.Structure):
    """min_settings_t (api/cablegen.h:47-59)."""
    _fields_ = [("free_formation", C.c_bool), ("ignore_f", C.c_bool), ("cores", C.c_longlong),
                ("nox", C.c_longlong), ("bdir", C.c_char_p), ("initial", C.c_char_p),
                ("end_gen", C.c_longlong), ("tdir", C.c_char_p), ("winstates", C.c_char_p),
                ("end_solve", C.c_longlong), ("delete_boards", C.c_bool)]


class SArr(C.Structure):
    _fields_ = [("valid", C.c_bool), ("bp", C.POINTER(C.c_uint64)), ("size", C.c_size_t)]


class Table(C.Structure):
    _fields_ = [("key", SArr), ("value", SArr)]


def load_ref():
    os.environ.setdefault("XDG_CONFIG_HOME", tempfile.mkdtemp())
    ref = C.CDLL(REF_LIB)
    ref.get_settings_min.restype = C.POINTER(MinSettings)
    for f in ("canonicalize_b", "rotate_clockwise", "flip"):
        getattr(ref, f).argtypes = [C.POINTER(C.c_uint64)]
    ref.movedir_unstable.argtypes = [C.POINTER(C.c_uint64), C.c_int]
    ref.movedir_unstable.restype = C.c_bool
    ref.movedir.argtypes = [C.POINTER(C.c_uint64), C.c_int]
    ref.movedir.restype = C.c_bool
    ref.prune_board.argtypes = [C.c_uint64, C.c_long, C.c_long, C.c_long]
    ref.prune_board.restype = C.c_bool
    ref.lookup.argtypes = [C.c_uint64, C.POINTER(Table), C.c_bool]
    ref.lookup.restype = C.c_double
    ref.cmpbrd.argtypes = [C.c_uint64, C.c_uint64]
    ref.cmpbrd.restype = C.c_bool
    ref.get_sum.argtypes = [C.c_uint64]
    ref.get_sum.restype = C.c_int
    ref.expectimax.argtypes = [C.c_uint64, C.POINTER(Table), C.POINTER(Table), C.c_void_p, C.c_char, C.c_bool]
    ref.expectimax.restype = C.c_double
    ref.set_log_level.argtypes = [C.c_int]
    ref.set_log_level(5)
    return ref


def random_boards(rng, n):
    """Boards with a realistic mix: 0xf formation cells, empties and tiles 1..13."""
    out = np.empty(n, dtype=np.uint64)
    for i in range(n):
        b = 0
        kind = rng.integers(0, 3)
        for c in range(16):
            r = rng.random()
            if kind == 0:
                e = int(rng.integers(0, 16))
            elif r < 0.35:
                e = 0
            elif r < 0.5:
                e = 0xF
            else:
                e = int(rng.integers(1, 11))
            b |= e << (60 - 4 * c)
        out[i] = b
    return out


def cmd_units(args):
    ref = load_ref()
    ms = ref.get_settings_min().contents
    rng = np.random.default_rng(configs.SEED)
    store = os.path.join(HERE, "units")
    os.makedirs(store, exist_ok=True)
    boards = random_boards(rng, args.n)
    boards.tofile(os.path.join(store, "boards.u64"))
    canon = np.empty_like(boards)
    for i, b in enumerate(boards):
        x = C.c_uint64(int(b))
        ref.canonicalize_b(C.byref(x))
        canon[i] = x.value
    canon.tofile(os.path.join(store, "canon.u64"))
    # movedir_unstable / movedir for all four settings combinations
    meta = {"n": int(args.n), "settings": []}
    for ff in (0, 1):
        for ig in (0, 1):
            ms.free_formation, ms.ignore_f = bool(ff), bool(ig)
            ref.generate_lut()
            lut = np.frombuffer((C.c_uint16 * (2 * 65536)).in_dll(ref, "_move_lut"), dtype=np.uint16).copy()
            locked = np.frombuffer((C.c_bool * (2 * 65536)).in_dll(ref, "_locked_lut"), dtype=np.uint8).copy()
            tag = f"ff{ff}_ig{ig}"
            h = hashlib.sha256(lut.tobytes() + locked.tobytes()).hexdigest()
            mv = np.zeros((len(boards), 4), dtype=np.uint64)
            ok = np.zeros((len(boards), 4), dtype=np.uint8)
            mvs = np.zeros((len(boards), 4), dtype=np.uint64)
            oks = np.zeros((len(boards), 4), dtype=np.uint8)
            for i, b in enumerate(boards):
                for d in range(4):
                    x = C.c_uint64(int(b))
                    ok[i, d] = ref.movedir_unstable(C.byref(x), d)
                    mv[i, d] = x.value
                    y = C.c_uint64(int(b))
                    oks[i, d] = ref.movedir(C.byref(y), d)
                    mvs[i, d] = y.value
            mv.tofile(os.path.join(store, f"move_unstable_{tag}.u64"))
            ok.tofile(os.path.join(store, f"move_unstable_ok_{tag}.u8"))
            mvs.tofile(os.path.join(store, f"move_stable_{tag}.u64"))
            oks.tofile(os.path.join(store, f"move_stable_ok_{tag}.u8"))
            meta["settings"].append({"tag": tag, "lut_sha256": h})
    ms.free_formation, ms.ignore_f = False, False
    ref.generate_lut()
    # prune_board over a grid of parameters
    params = [(58, 5, 6), (64, 6, 6), (200, 5, 6), (0, 0, 0), (30, 3, 4), (120, 8, 7)]
    pr = np.zeros((len(params), len(boards)), dtype=np.uint8)
    for j, (stsl, ltc, sl) in enumerate(params):
        for i, b in enumerate(boards):
            pr[j, i] = ref.prune_board(int(b), stsl, ltc, sl)
    pr.tofile(os.path.join(store, "prune.u8"))
    meta["prune_params"] = params
    # cmpbrd against sparse patterns
    pats = np.array([int(boards[i]) & int(rng.integers(0, 1 << 63)) & 0xF0F00F000F00F00F
                     for i in range(64)], dtype=np.uint64)
    cm = np.zeros((64, 256), dtype=np.uint8)
    for j, w in enumerate(pats):
        for i in range(256):
            cm[j, i] = ref.cmpbrd(int(boards[i]), int(w))
    pats.tofile(os.path.join(store, "cmpbrd_patterns.u64"))
    cm.tofile(os.path.join(store, "cmpbrd.u8"))
    sums = np.array([ref.get_sum(int(b)) for b in boards], dtype=np.int32)
    sums.tofile(os.path.join(store, "get_sum.i32"))
    # lookup: sorted unique keys with values, queries that hit and miss
    keys = np.unique(canon)
    vals = rng.random(len(keys))
    queries = np.concatenate([boards[: len(boards) // 2], rng.integers(0, 1 << 63, len(boards) // 2, dtype=np.uint64)])
    t = Table()
    t.key = SArr(True, keys.ctypes.data_as(C.POINTER(C.c_uint64)), len(keys))
    t.value = SArr(True, vals.view(np.uint64).ctypes.data_as(C.POINTER(C.c_uint64)), len(keys))
    res = np.array([ref.lookup(int(q), C.byref(t), True) for q in queries], dtype=np.float64)
    res_nc = np.array([ref.lookup(int(q), C.byref(t), False) for q in queries], dtype=np.float64)
    keys.tofile(os.path.join(store, "lookup_keys.u64"))
    vals.tofile(os.path.join(store, "lookup_vals.f64"))
    queries.tofile(os.path.join(store, "lookup_queries.u64"))
    res.tofile(os.path.join(store, "lookup_canon.f64"))
    res_nc.tofile(os.path.join(store, "lookup_nocanon.f64"))
    # expectimax over the two tables: successors drawn from the table keys
    ex = np.array([ref.expectimax(int(b), C.byref(t), C.byref(t), None, b"\0", False) for b in boards[:2048]],
                  dtype=np.float64)
    ex.tofile(os.path.join(store, "expectimax.f64"))
    with open(os.path.join(store, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("units written:", store, "boards:", len(boards), "lookup keys:", len(keys),
          "hits:", int((res != 0).sum()))


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run")
    r.add_argument("workload")
    r.add_argument("--cores", type=int, default=os.cpu_count())
    r.add_argument("--end", type=int, default=None)
    r.add_argument("--keep", default=None, help="keep the reference's files in this directory")
    r.add_argument("--no-solve", action="store_true")
    r.add_argument("--reuse", action="store_true", help="reuse the boards already generated in --keep")
    sub.add_parser("cli")
    u = sub.add_parser("units")
    u.add_argument("--n", type=int, default=4096)
    a = ap.parse_args()
    if not os.path.exists(REF_CLI):
        sys.exit("build the reference first: make -C oracle all")
    {"run": cmd_run, "units": cmd_units, "cli": cmd_cli}[a.cmd](a)


if __name__ == "__main__":
    main()
