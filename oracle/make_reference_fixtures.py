"""Generate golden fixtures by running the REFERENCE library (test infrastructure).

Two steps:

  python oracle/make_reference_fixtures.py run  --out DIR [--only PART ...]   (with a GPU)
      builds nothing; needs oracle/_ref/ref_driver (``make -C oracle ref``).  Writes the
      stage inputs, runs the reference driver on them, on the parity sequences and on the
      colour-lookup probes and the rotational predictor / Lax-Wendroff cases, and leaves raw
      outputs in DIR.  PART: stages, norm, upmap, cases, wheelidx, rotation, long (default:
      all).  "long" streams the long cases (1000 frames of 2048x1088) through the reference
      one frame at a time and keeps a sha256 of every frame's flow.

  python oracle/make_reference_fixtures.py pack --raw DIR
      packs DIR into the small committed fixtures under tests/golden/.

The parity sequences are regenerated from seeds by flowfilter_b200.synthetic; the
fixtures carry a sha256 of the frames so a drifting generator is detected.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "optical-flow-filter_b200"))

from flowfilter_b200 import synthetic  # noqa: E402

sys.path.insert(0, ROOT)
from oracle import display_oracle  # noqa: E402

DRIVER = os.path.join(HERE, "_ref", "ref_driver")
GOLDEN = os.path.join(ROOT, "tests", "golden")

# stage inputs: odd sizes so the pyramid's integer halving and the edges are exercised
STAGE_H, STAGE_W = 53, 70

# parity sequences (name -> parameters).  levels 0 = single-level FlowFilter.
CASES = {
    "constant_320x240_L1": dict(seq="constant", frames=100, levels=0, maxflow=4.0,
                                gamma=[10.0], smooth=[1], dump=[1, 2, 10, 50, 99]),
    "rotzoom_640x480_L2": dict(seq="rotzoom", frames=300, levels=2, maxflow=4.0,
                               gamma=[10.0, 50.0], smooth=[2, 4], dump=[1, 10, 100, 299]),
    "bumps_2048x1088_L3": dict(seq="bumps", frames=60, levels=3, maxflow=4.0,
                               gamma=[5.0, 20.0, 50.0], smooth=[1, 2, 4], dump=[1, 20, 59]),
    "odd_77x61_L1": dict(seq="constant", frames=40, levels=0, maxflow=2.5, gamma=[3.0],
                         smooth=[2], dump=list(range(0, 40, 3)) + [39],
                         kw=dict(height=61, width=77, sigma=1.2, seed=11, flow=(1.3, 0.6))),
    "odd_150x98_L3": dict(seq="rotzoom", frames=40, levels=3, maxflow=3.0,
                          gamma=[4.0, 9.0, 30.0], smooth=[1, 3, 2], dump=list(range(0, 40, 3)) + [39],
                          kw=dict(height=98, width=150, sigma=1.0, seed=12, deg_per_frame=1.5,
                                  zoom_per_frame=1.01)),
    "small_96x64_L2": dict(seq="bumps", frames=40, levels=2, maxflow=5.0, gamma=[2.0, 25.0],
                           smooth=[3, 1], dump=list(range(0, 40, 3)) + [39],
                           kw=dict(height=64, width=96, sigma=1.0, seed=13, n_bumps=3,
                                   bump_sigma=20.0, amp=2.0, sensor_noise=2.0)),
}

# colour-lookup probes: (maxflow, seed) per case
WHEEL_CASES = [(1.0, 31), (4.0, 32), (0.3, 33), (7.5, 34)]

# Lax-Wendroff propagation cases: (H, W, depth, iterations, seed); iterations 0 = never set
LW_CASES = [(37, 53, 1, 1, 41), (37, 53, 1, 4, 42), (37, 53, 4, 3, 43), (64, 80, 1, 0, 44), (64, 80, 4, 1, 45),
            (20, 33, 4, 8, 46), (96, 128, 1, 2, 47)]
# rotational predictor cases: (H, W, depth, focal, sensorH, sensorW, wx, wy, wz, iterations, seed)
ROT_CASES = [(48, 64, 1, 0.004, 0.0036, 0.0048, 0.02, -0.015, 0.04, 2, 51),
             (45, 61, 4, 0.0035, 0.003, 0.004, -0.03, 0.01, -0.02, 3, 52),
             (60, 90, 1, 0.006, 0.0045, 0.0068, 0.0, 0.0, 0.1, 0, 53),
             (33, 40, 4, 0.002, 0.0024, 0.0032, 0.05, 0.05, 0.0, 1, 54)]

FULL_LIMIT = 64 * 128  # dumps up to this many pixels are stored whole

# long sequences: every frame's flow is hashed (sha256 of the float32 (H, W, 2) flow) and a few
# frames are kept subsampled; frames are generated and streamed through the reference one at a time
LONG_CASES = {
    "bumps_2048x1088_L3_1000": dict(seq="bumps", frames=1000, levels=3, maxflow=4.0,
                                    gamma=[5.0, 20.0, 50.0], smooth=[1, 2, 4], keep=[500, 999]),
}


def stage_inputs(seed: int = 5) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    h, w = STAGE_H, STAGE_W
    hc, wc = h // 2, w // 2
    return {
        "img_u8": rng.integers(0, 256, size=(h, w), dtype=np.uint8),
        "img_f32": rng.uniform(0, 1, size=(h, w)).astype(np.float32),
        "flow": (rng.normal(0, 1.5, size=(h, w, 2))).astype(np.float32),
        "scalar": rng.uniform(0, 1, size=(h, w)).astype(np.float32),
        "vector": (rng.normal(0, 0.8, size=(h, w, 2))).astype(np.float32),
        "a0": rng.uniform(0, 1, size=(h, w)).astype(np.float32),
        "grad": (rng.normal(0, 0.05, size=(h, w, 2))).astype(np.float32),
        "a0old": rng.uniform(0, 1, size=(h, w)).astype(np.float32),
        "coarse": (rng.normal(0, 1.0, size=(hc, wc, 2))).astype(np.float32),
    }


def case_frames(case: dict) -> np.ndarray:
    return synthetic.sequence(case["seq"], frames=case["frames"], **case.get("kw", {}))


def long_frames(case: dict):
    """The frames of a long case one at a time (uint8 (H, W))."""
    assert case["seq"] == "bumps"
    return synthetic.iter_bumps(frames=case["frames"], **case.get("kw", {}))


def run_long(out: str) -> None:
    """Streams each long case through the reference (ref_driver filterpipe) and writes
    long_NAME.npz: per-frame sha256 digests of the flow and the kept frames subsampled."""
    import threading

    for name, case in LONG_CASES.items():
        frames = long_frames(case)
        first = next(frames)
        h, w = first.shape
        cmd = [DRIVER, "filterpipe", str(h), str(w), str(case["levels"]), repr(case["maxflow"]),
               ",".join(repr(g) for g in case["gamma"]), ",".join(str(s) for s in case["smooth"])]
        proc = subprocess.Popen(cmd, stdin=subprocess.PIPE, stdout=subprocess.PIPE)
        frame_sha = hashlib.sha256()

        def feed():
            try:
                proc.stdin.write(first.tobytes())
                frame_sha.update(first.tobytes())
                for f in frames:
                    proc.stdin.write(f.tobytes())
                    frame_sha.update(f.tobytes())
            finally:
                proc.stdin.close()

        th = threading.Thread(target=feed)
        th.start()
        fsz = h * w * 8
        digests, kept = [], {}
        rows, cols = subsample_rows_cols(h, w)
        for t in range(case["frames"]):
            buf = proc.stdout.read(fsz)
            if len(buf) != fsz:
                raise RuntimeError(f"{name}: reference stopped at frame {t}")
            digests.append(hashlib.sha256(buf).digest())
            if t in case["keep"]:
                kept[t] = np.frombuffer(buf, np.float32).reshape(h, w, 2)[rows][:, cols].copy()
        th.join()
        if proc.wait() != 0:
            raise RuntimeError(f"{name}: reference driver failed")
        # the frames this run shares with a short parity case must give that case's flows
        short = os.path.join(GOLDEN, "ref_case_bumps_2048x1088_L3.npz")
        if name.startswith("bumps_2048x1088_L3") and os.path.exists(short):
            m = json.loads(bytes(np.load(short)["meta"]).decode())
            for t, want in zip(m["dump"], m["flow_sha256"]):
                if digests[t].hex() != want:
                    raise RuntimeError(f"{name}: frame {t} differs from the short reference run")
        meta = dict(case, name=name, frames_sha256=frame_sha.hexdigest(), layout="subsampled")
        np.savez_compressed(os.path.join(out, f"long_{name}.npz"),
                            digests=np.frombuffer(b"".join(digests), np.uint8).reshape(-1, 32),
                            keep=np.array(case["keep"], np.int64), rows=rows, cols=cols,
                            flow=np.stack([kept[t] for t in case["keep"]]),
                            meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8))


def lw_inputs(h: int, w: int, depth: int, seed: int):
    """(flow (H, W, 2), image (H, W) or (H, W, 4)) float32 for a Lax-Wendroff case: a smooth
    flow of a few pixels with some large values, a noisy image."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    flow = np.stack([2.0 * np.sin(xx / 7.0 + yy / 11.0), 1.5 * np.cos(yy / 5.0 - xx / 13.0)], -1)
    flow += rng.normal(0, 0.3, flow.shape)
    flow.reshape(-1, 2)[rng.integers(0, h * w, 8)] = rng.uniform(-9, 9, (8, 2))
    img = rng.random((h, w) if depth == 1 else (h, w, depth))
    return flow.astype(np.float32), img.astype(np.float32)


def rot_image(h: int, w: int, depth: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.random((h, w) if depth == 1 else (h, w, depth)).astype(np.float32)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(out: str, only=None) -> None:
    parts = set(only or ["stages", "norm", "upmap", "cases", "wheelidx", "rotation", "long"])
    os.makedirs(out, exist_ok=True)
    if "long" in parts:
        run_long(out)
    if "stages" in parts:
        sin = os.path.join(out, "stage_in")
        sout = os.path.join(out, "stage_out")
        os.makedirs(sin, exist_ok=True)
        os.makedirs(sout, exist_ok=True)
        for k, v in stage_inputs().items():
            np.save(os.path.join(sin, k + ".npy"), v)
        subprocess.run([DRIVER, "stages", sin, sout], check=True)
    if "norm" in parts:
        subprocess.run([DRIVER, "norm", os.path.join(out, "norm.npy")], check=True)
    if "upmap" in parts:
        subprocess.run([DRIVER, "upmap", os.path.join(out, "upmap.txt"), "4200"], check=True)
    if "wheelidx" in parts:
        for k, (m, seed) in enumerate(WHEEL_CASES):
            fpath = os.path.join(out, f"wheel_flows_{k}.npy")
            np.save(fpath, display_oracle.probe_flows(m, seed))
            subprocess.run([DRIVER, "wheelidx", fpath, repr(m), os.path.join(out, f"wheel_idx_{k}.npy")], check=True)
    if "rotation" in parts:
        for k, (h, w, d, it, seed) in enumerate(LW_CASES):
            flow, img = lw_inputs(h, w, d, seed)
            fp, ip = os.path.join(out, f"lw_flow_{k}.npy"), os.path.join(out, f"lw_img_{k}.npy")
            np.save(fp, flow)
            np.save(ip, img)
            subprocess.run([DRIVER, "lw", fp, ip, str(it), os.path.join(out, f"lw_out_{k}.npy")], check=True)
        for k, (h, w, d, focal, sh, sw, wx, wy, wz, it, seed) in enumerate(ROT_CASES):
            ip = os.path.join(out, f"rot_img_{k}.npy")
            np.save(ip, rot_image(h, w, d, seed))
            subprocess.run([DRIVER, "rotation", ip, repr(focal), repr(sh), repr(sw), repr(wx), repr(wy), repr(wz),
                            str(it), os.path.join(out, f"rot_flow_{k}.npy"), os.path.join(out, f"rot_pred_{k}.npy")],
                           check=True)
    if "cases" not in parts:
        return
    tmp = os.environ.get("TMPDIR", "/tmp")
    for name, case in CASES.items():
        frames = case_frames(case)
        fpath = os.path.join(tmp, f"frames_{name}.npy")
        np.save(fpath, frames)
        raw = os.path.join(tmp, f"flow_{name}.npy")
        timing = os.path.join(out, f"timing_{name}.csv")
        cmd = [DRIVER, "filter", fpath, raw, str(case["levels"]), repr(case["maxflow"]),
               ",".join(repr(g) for g in case["gamma"]), ",".join(str(s) for s in case["smooth"]),
               ",".join(str(d) for d in case["dump"]), timing]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        flows = np.load(raw)
        pack_flows(os.path.join(out, f"case_{name}.npz"), name, case, frames, flows)
        os.remove(fpath)
        os.remove(raw)


def subsample_rows_cols(h: int, w: int) -> tuple[np.ndarray, np.ndarray]:
    # every 5th row and 7th column, plus the last row/column so the edges are pinned
    rows = np.unique(np.concatenate([np.arange(0, h, 5), [1, 2, h - 3, h - 2, h - 1]]))
    cols = np.unique(np.concatenate([np.arange(0, w, 7), [1, 2, w - 3, w - 2, w - 1]]))
    return rows, cols


def pack_flows(path: str, name: str, case: dict, frames: np.ndarray, flows: np.ndarray) -> None:
    t, h, w = frames.shape
    meta = dict(case)
    meta["name"] = name
    meta["frames_sha256"] = sha(frames)
    meta["flow_sha256"] = [sha(f) for f in flows]
    arrays = {}
    if h * w <= FULL_LIMIT:
        arrays["flow"] = flows
        meta["layout"] = "full"
    else:
        rows, cols = subsample_rows_cols(h, w)
        arrays["rows"] = rows
        arrays["cols"] = cols
        arrays["flow"] = flows[:, rows][:, :, cols]
        meta["layout"] = "subsampled"
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrays)


def pack(raw: str) -> None:
    os.makedirs(GOLDEN, exist_ok=True)
    # stage goldens: inputs are regenerated from the seed, outputs stored whole
    sout = os.path.join(raw, "stage_out")
    if os.path.isdir(sout):
        outs = {f[:-4]: np.load(os.path.join(sout, f)) for f in sorted(os.listdir(sout)) if f.endswith(".npy")}
        ins = stage_inputs()
        np.savez_compressed(os.path.join(GOLDEN, "ref_stages.npz"),
                            inputs_sha256=np.frombuffer(json.dumps({k: sha(v) for k, v in ins.items()}).encode(),
                                                        np.uint8),
                            **outs)
    if os.path.exists(os.path.join(raw, "norm.npy")):
        np.save(os.path.join(GOLDEN, "ref_norm_u8.npy"), np.load(os.path.join(raw, "norm.npy")))
    if os.path.exists(os.path.join(raw, "upmap.txt.detail.npy")):
        np.save(os.path.join(GOLDEN, "ref_upmap_detail.npy"), np.load(os.path.join(raw, "upmap.txt.detail.npy")))
    if os.path.exists(os.path.join(raw, "wheel_idx_0.npy")):
        # texel picked per pixel by the reference lookup: column (R), row (G)
        idx = np.stack([np.load(os.path.join(raw, f"wheel_idx_{k}.npy")) for k in range(len(WHEEL_CASES))])
        assert (idx[..., 2] == 0).all() and (idx[..., 3] == 255).all()
        flows_sha = [sha(display_oracle.probe_flows(m, seed)) for m, seed in WHEEL_CASES]
        np.savez_compressed(os.path.join(GOLDEN, "ref_flow_to_color.npz"), col=idx[..., 0], row=idx[..., 1],
                            maxflow=np.array([m for m, _ in WHEEL_CASES], np.float32),
                            seed=np.array([s for _, s in WHEEL_CASES], np.int64),
                            flows_sha256=np.frombuffer(json.dumps(flows_sha).encode(), np.uint8))
    if os.path.exists(os.path.join(raw, "lw_out_0.npy")):
        arrays = {}
        shas = {}
        for k, (h, w, d, it, seed) in enumerate(LW_CASES):
            flow, img = lw_inputs(h, w, d, seed)
            shas[f"lw_{k}"] = [sha(flow), sha(img)]
            arrays[f"lw_out_{k}"] = np.load(os.path.join(raw, f"lw_out_{k}.npy"))
        for k, case in enumerate(ROT_CASES):
            h, w, d, seed = case[0], case[1], case[2], case[-1]
            shas[f"rot_{k}"] = [sha(rot_image(h, w, d, seed))]
            arrays[f"rot_flow_{k}"] = np.load(os.path.join(raw, f"rot_flow_{k}.npy"))
            arrays[f"rot_pred_{k}"] = np.load(os.path.join(raw, f"rot_pred_{k}.npy"))
            arrays[f"rot_cam_{k}"] = np.load(os.path.join(raw, f"rot_flow_{k}.npy.cam.npy"))
        np.savez_compressed(os.path.join(GOLDEN, "ref_rotation.npz"),
                            inputs_sha256=np.frombuffer(json.dumps(shas).encode(), np.uint8), **arrays)
    for name in LONG_CASES:
        src = os.path.join(raw, f"long_{name}.npz")
        if os.path.exists(src):
            with open(src, "rb") as fi, open(os.path.join(GOLDEN, f"ref_long_{name}.npz"), "wb") as fo:
                fo.write(fi.read())
    for name in CASES:
        src = os.path.join(raw, f"case_{name}.npz")
        if os.path.exists(src):
            with open(src, "rb") as fi, open(os.path.join(GOLDEN, f"ref_case_{name}.npz"), "wb") as fo:
                fo.write(fi.read())


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run")
    r.add_argument("--out", required=True)
    r.add_argument("--only", nargs="*", default=None)
    p = sub.add_parser("pack")
    p.add_argument("--raw", required=True)
    a = ap.parse_args()
    if a.cmd == "run":
        run(a.out, a.only)
    else:
        pack(a.raw)


if __name__ == "__main__":
    main()
