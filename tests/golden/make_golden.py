"""Extract the known-answer values from the reference's recorded stdout runs.

Reads ``sim_output_*_gpu.txt`` of the cudaturbo reference (recorded on an RTX 3090) and writes
``reference_stdout.json`` beside this script: the PAO initial-condition statistics, the
NEXTDT-init line and every ``ITERATION`` line (T, DT, CN, CFLM, SIG) of each run.  The JSON is
committed; this script is only re-run when the reference changes:

    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import re
import sys

RUNS = [
    "sim_output_512_1001_gpu.txt",
    "sim_output_4096_501_gpu.txt",
    "sim_output_16384_21_gpu.txt",
    "sim_output_16384_101_gpu.txt",
]

STAT_RE = re.compile(r"^ ([A-Za-z0-9/\. ]+?)\s*=\s*([-+0-9.eE]+)\s*$")
HEAD_RE = re.compile(r"N=(\d+), Re=(\d+), K0=(\d+), STEPS=(\d+), CFL=([0-9.]+), UPDATE=(\d+)")
INIT_RE = re.compile(r"\[NEXTDT INIT\] CFLM=\s*([-0-9.eE]+)\s+DT=\s*([-0-9.eE]+)\s+CN=\s*([-0-9.eE]+)")
ITER_RE = re.compile(r"ITERATION\s+(\d+) T=([-0-9.eE]+) DT=([-0-9.eE]+) CN=([-0-9.eE]+) "
                     r"CFLM=([-0-9.eE]+) .* SIG=(\d+)")


def parse(path):
    run = {"file": os.path.basename(path), "pao": {}, "iterations": []}
    with open(path) as f:
        for line in f:
            m = HEAD_RE.search(line)
            if m and "N" not in run:
                run.update(N=int(m[1]), Re=float(m[2]), K0=float(m[3]), STEPS=int(m[4]),
                           CFL=float(m[5]), UPDATE=int(m[6]))
                continue
            m = INIT_RE.search(line)
            if m:
                run["nextdt_init"] = {"CFLM": float(m[1]), "DT": float(m[2]), "CN": float(m[3])}
                continue
            m = ITER_RE.search(line)
            if m:
                run["iterations"].append({"it": int(m[1]), "T": float(m[2]), "DT": float(m[3]),
                                          "CN": float(m[4]), "CFLM": float(m[5]),
                                          "SIG": int(m[6])})
                continue
            if line.startswith(" PAO seed"):
                run["pao_seed"] = int(line.split("=")[1])
                continue
            m = STAT_RE.match(line.rstrip("\n"))
            if m and "cuFFT" not in line and "dnsCudaCreate" not in line:
                run["pao"][m[1].strip()] = m[2]
    return run


def main():
    # the reference checkout: first argument, else $REF, else the build container's copy
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF", "/root/reference")
    out = {"source": "cudaturbo reference stdout (RTX 3090 runs)", "runs": []}
    for name in RUNS:
        out["runs"].append(parse(os.path.join(ref, name)))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_stdout.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main()
