"""Generate golden vectors from the reference's own code (run on a GPU host).

Runs the reference binaries and libraries built by ``oracle/Makefile`` into
``oracle/_ref/`` on seeded inputs and records their outputs:

* ``mappingV15``       -- the reference GPU uint16 mapping
                          (mapping/nv/mappingV15_fused_uint16.cu), file in/out;
* ``mappingV9``        -- the reference GPU uint32 escape mapping
                          (mapping/nv/mappingV9_fuse.cu), file in/out;
* ``mappingV12``       -- the reference GPU uint16 mapping with the V12 merged
                          layout (mapping/nv/mappingV12_bit-adm-thrust-prefixsum.cu),
                          file in/out;
* ``ref_ans_driver``   -- the reference GPU rANS codec (include/ans) through
                          ansEncode/ansDecode;
* ``libref_adm_cpu.so``-- the reference CPU mapping (mapping/cpu/mappingcpuV2.cpp),
                          run with one OpenMP thread (its lane-length update
                          races when a warp's lanes span OpenMP chunks), in
                          the V15 layout and in its own g + 1 header layout.

Only inputs on which the reference is defined are used: N a multiple of 1024
(the GPU mappers read and write whole vectors), more than 524,288 uint16
values (V15 then takes its thrust path; its look-back path reads an
uninitialised shared variable), lane bit streams under 256 bits (the V15
lane buffer), uint32 group sums below 2^32, and rANS blocks whose output
stays under the reference's 5,120-byte block slot.

V12 is run only on N a multiple of 1,024: its decompress kernel writes whole
1,024-element blocks, past its output buffer for other N.

Usage (from the repository root; the GPU kinds on the GPU host):
    python tests/golden/make_golden.py <outdir> [--only kind,kind,...]
    python tests/golden/make_golden.py --merge <outdir>
The first writes ``<outdir>/manifest.json`` and small ``.bin`` files for the
selected kinds (all by default); the second merges such a directory into the
committed copies in tests/golden/.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mans_b200 import workloads as W  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
SMALL = 1 << 16  # store full bytes for outputs up to this size


def sha(b: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(b).view(np.uint8).tobytes()).hexdigest()


def gen(spec: dict) -> np.ndarray:
    g = spec["gen"]
    n = spec["n"]
    seed = spec["seed"]
    if g == "laplace_u16":
        return W.laplace_u16(n, seed, b=spec.get("b", 40.0))
    if g == "gradient_u16":
        return W.gradient_u16(n, seed)
    if g == "volume_u16":
        return W.volume_u16(n, seed)
    if g == "detector_u32":
        return W.detector_u32(n, seed)
    if g.startswith("bytes_"):
        return W.random_bytes(n, seed, g[len("bytes_"):])
    if g == "adm_u16_of":
        return O.adm_u16_map(gen(spec["of"]))
    if g == "adm_u32_of":
        return O.adm_u32_map(gen(spec["of"]))
    raise ValueError(g)


def max_lane_bits_u16(x: np.ndarray) -> int:
    """Longest lane bit stream of the uint16 mapping (16 elements per lane)."""
    g = x.reshape(-1, 512).astype(np.int64)
    c = g.sum(axis=1) // 512
    d = np.abs(g - c[:, None])
    k = np.maximum(1, (d + 125) // 126)
    return int(k.reshape(-1, 16).sum(axis=1).max())


def run(cmd: list[str]) -> str:
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed ({r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return r.stdout


def record(entry: dict, arr: np.ndarray, outdir: str, key: str) -> None:
    entry[key + "_sha256"] = sha(arr)
    entry[key + "_size"] = int(arr.size)
    if arr.size <= SMALL:
        fn = f"{entry['name']}.{key}.bin"
        arr.astype(np.uint8).tofile(os.path.join(outdir, fn))
        entry[key + "_file"] = fn


def ans_cases():
    cases = []
    for kind, sizes in [("skewed", [0, 1, 31, 32, 33, 4095, 4096, 4097, 65536, 100000]),
                        ("uniform", [5000, 65536]), ("single", [1000, 8192]),
                        ("two", [12345]), ("sparse", [70000])]:
        for i, n in enumerate(sizes):
            for p in (9, 10, 11):
                cases.append({"name": f"ans_{kind}_{n}_p{p}", "kind": "ans", "prob_bits": p,
                              "input": {"gen": f"bytes_{kind}", "n": n, "seed": 100 + i}})
    c1 = {"gen": "laplace_u16", "n": W.C1_N, "seed": 1}
    for p in (9, 10, 11):
        cases.append({"name": f"ans_adm_c1_p{p}", "kind": "ans", "prob_bits": p,
                      "input": {"gen": "adm_u16_of", "n": 0, "seed": 0, "of": c1}})
    vol = {"gen": "volume_u16", "n": 1 << 20, "seed": 4}
    cases.append({"name": "ans_adm_volume_p10", "kind": "ans", "prob_bits": 10,
                  "input": {"gen": "adm_u16_of", "n": 0, "seed": 0, "of": vol}})
    det = {"gen": "detector_u32", "n": 1 << 20, "seed": 2}
    cases.append({"name": "ans_adm32_detector_p10", "kind": "ans", "prob_bits": 10,
                  "input": {"gen": "adm_u32_of", "n": 0, "seed": 0, "of": det}})
    return cases


def v15_cases():
    return [
        {"name": "v15_c1", "kind": "adm_u16_gpu", "input": {"gen": "laplace_u16", "n": W.C1_N, "seed": 1}},
        {"name": "v15_gradient", "kind": "adm_u16_gpu", "input": {"gen": "gradient_u16", "n": 1 << 20, "seed": 3}},
        {"name": "v15_volume", "kind": "adm_u16_gpu", "input": {"gen": "volume_u16", "n": 1 << 20, "seed": 4}},
        {"name": "v15_wide", "kind": "adm_u16_gpu", "input": {"gen": "laplace_u16", "n": 525312, "seed": 9, "b": 600.0}},
    ]


def v9_cases():
    return [
        {"name": "v9_detector", "kind": "adm_u32_gpu", "input": {"gen": "detector_u32", "n": 1 << 20, "seed": 2}},
        {"name": "v9_detector_small", "kind": "adm_u32_gpu", "input": {"gen": "detector_u32", "n": 1 << 16, "seed": 5}},
    ]


def cpu_cases():
    out = []
    for i, n in enumerate([1, 7, 8, 15, 16, 17, 100, 511, 512, 513, 1000, 4095, 4096, 4097, 20000]):
        out.append({"name": f"cpuv2_laplace_{n}", "kind": "adm_u16_cpu",
                    "input": {"gen": "laplace_u16", "n": n, "seed": 200 + i, "b": 300.0}})
    out.append({"name": "cpuv2_wide_3000", "kind": "adm_u16_cpu",
                "input": {"gen": "laplace_u16", "n": 3000, "seed": 250, "b": 4000.0}})
    return out


def cpu_native_cases():
    out = []
    for i, n in enumerate([1, 16, 511, 512, 513, 1040, 4097, 20000, 70001]):
        out.append({"name": f"cpuv2native_laplace_{n}", "kind": "adm_u16_cpu_native",
                    "input": {"gen": "laplace_u16", "n": n, "seed": 400 + i, "b": 300.0}})
    out.append({"name": "cpuv2native_c1", "kind": "adm_u16_cpu_native",
                "input": {"gen": "laplace_u16", "n": W.C1_N, "seed": 1}})
    return out


def v12_cases():
    return [
        {"name": "v12_laplace_1024", "kind": "adm_u16_v12_gpu",
         "input": {"gen": "laplace_u16", "n": 1024, "seed": 500, "b": 300.0}},
        {"name": "v12_laplace_65536", "kind": "adm_u16_v12_gpu",
         "input": {"gen": "laplace_u16", "n": 65536, "seed": 501, "b": 300.0}},
        {"name": "v12_gradient", "kind": "adm_u16_v12_gpu",
         "input": {"gen": "gradient_u16", "n": 1 << 20, "seed": 3}},
        {"name": "v12_c1", "kind": "adm_u16_v12_gpu",
         "input": {"gen": "laplace_u16", "n": W.C1_N, "seed": 1}},
    ]


KINDS = ("adm_u16_cpu", "adm_u16_cpu_native", "adm_u16_gpu", "adm_u16_v12_gpu", "adm_u32_gpu", "ans")


def merge(src: str) -> None:
    """Merge the cases of src/manifest.json into the committed golden set."""
    import shutil
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(src, "manifest.json")) as f:
        new = json.load(f)
    path = os.path.join(here, "manifest.json")
    with open(path) as f:
        old = json.load(f)
    names = {c["name"] for c in new}
    merged = [c for c in old if c["name"] not in names] + new
    for c in new:
        for k, v in c.items():
            if k.endswith("_file"):
                shutil.copy(os.path.join(src, v), os.path.join(here, v))
    with open(path, "w") as f:
        json.dump(merged, f, indent=1)
    print(f"merged {len(new)} cases; {len(merged)} in total")


def main(outdir: str, only=KINDS) -> None:
    os.makedirs(outdir, exist_ok=True)
    manifest = []
    tmp = tempfile.mkdtemp()
    # --- reference CPU mapping in its own layout (g + 1 prefix words)
    for c in (cpu_native_cases() if "adm_u16_cpu_native" in only else []):
        x = gen(c["input"])
        r = O.RefAdmCpu(x)
        r.compress()
        m = r.merged(False)
        r.decompress()
        c["ref_roundtrip"] = bool(np.array_equal(r.recovered(), x))
        record(c, m, outdir, "ref")
        r.close()
        manifest.append(c)
    # --- reference GPU uint16 mapping, V12 layout
    for c in (v12_cases() if "adm_u16_v12_gpu" in only else []):
        x = gen(c["input"])
        assert x.size % 1024 == 0 and max_lane_bits_u16(x) <= 256, c["name"]
        fi = os.path.join(tmp, "in.u2")
        fo = os.path.join(tmp, "out.adm")
        x.tofile(fi)
        log = run([os.path.join(REF, "mappingV12"), fi, fo, "uint16"])
        m = np.fromfile(fo, np.uint8)
        c["ref_log_pass"] = "Pass error check" in log
        record(c, m, outdir, "ref")
        manifest.append(c)
    # --- reference CPU mapping (one thread)
    for c in (cpu_cases() if "adm_u16_cpu" in only else []):
        x = gen(c["input"])
        r = O.RefAdmCpu(x)
        r.compress()
        m = r.merged(True)
        r.decompress()
        c["ref_roundtrip"] = bool(np.array_equal(r.recovered(), x))
        if not c["ref_roundtrip"]:
            c["ref_defined"] = False
            c["note"] = ("lane bit streams exceed the reference lane buffer (32 bytes); "
                         "the reference fails its own round trip")
        record(c, m, outdir, "ref")
        r.close()
        manifest.append(c)
    # --- reference GPU uint16 mapping
    for c in (v15_cases() if "adm_u16_gpu" in only else []):
        x = gen(c["input"])
        assert max_lane_bits_u16(x) <= 256, c["name"]
        fi = os.path.join(tmp, "in.u2")
        fo = os.path.join(tmp, "out.adm")
        x.tofile(fi)
        log = run([os.path.join(REF, "mappingV15"), fi, fo])
        m = np.fromfile(fo, np.uint8)
        c["ref_log_pass"] = "Pass error check" in log
        record(c, m, outdir, "ref")
        manifest.append(c)
    # --- reference GPU uint32 mapping (records only)
    for c in (v9_cases() if "adm_u32_gpu" in only else []):
        x = gen(c["input"])
        fi = os.path.join(tmp, "in.u4")
        fo = os.path.join(tmp, "out.adm")
        x.tofile(fi)
        log = run([os.path.join(REF, "mappingV9"), fi, fo, "uint32"])
        m = np.fromfile(fo, np.uint8)
        c["ref_log_pass"] = "Pass error check" in log
        record(c, m, outdir, "ref")
        manifest.append(c)
    # --- reference GPU rANS
    for c in (ans_cases() if "ans" in only else []):
        x = gen(c["input"])
        _, bw = O.ans_encode(x, c["prob_bits"], with_block_words=True)
        if bw.size and int(bw.max()) * 2 > 5120 - 16:
            c["skipped"] = "a block exceeds the reference's 5,120-byte slot"
            manifest.append(c)
            continue
        fi = os.path.join(tmp, "in.bin")
        fs = os.path.join(tmp, "s.ans")
        fd = os.path.join(tmp, "d.bin")
        x.tofile(fi)
        log = run([os.path.join(REF, "ref_ans_driver"), str(c["prob_bits"]), fi, fs, fd])
        s = np.fromfile(fs, np.uint8)
        d = np.fromfile(fd, np.uint8)
        c["ref_roundtrip"] = bool(np.array_equal(d, x))
        c["input_sha256"] = sha(x)
        record(c, O.ans_mask(s), outdir, "ref")
        manifest.append(c)
    with open(os.path.join(outdir, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(f"wrote {len(manifest)} cases to {outdir}")


if __name__ == "__main__":
    args = sys.argv[1:]
    if args[:1] == ["--merge"]:
        merge(args[1])
    else:
        only = KINDS
        if "--only" in args:
            i = args.index("--only")
            only = tuple(args[i + 1].split(","))
            args = args[:i] + args[i + 2:]
        if not args:
            sys.exit("usage: make_golden.py OUTDIR [--only kinds] | --merge OUTDIR")
        main(args[0], only)
