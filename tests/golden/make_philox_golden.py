"""Writes philox_curand.json: cuRAND Philox4_32_10 outputs (curand_init(seed, subsequence,
offset) then curand4) for a few cases. Needs nvcc and a CUDA device:

    python tests/golden/make_philox_golden.py

cuRAND keys Philox with (lo32(seed), hi32(seed)) and starts the counter at
(lo32(offset/4), hi32(offset/4), lo32(subsequence), hi32(subsequence)), incrementing it by
one per curand4 call; the CPU test maps each case to that counter and compares."""
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "curand_philox")
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-o", exe,
                        os.path.join(HERE, "curand_philox.cu")], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    cases = [json.loads(line) for line in out.splitlines() if line.strip()]
    with open(os.path.join(HERE, "philox_curand.json"), "w") as f:
        json.dump(cases, f, indent=1)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
