"""Regenerates tests/golden/philox_curand.json on a CUDA GPU:
compiles philox_curand.cu (calls cuRAND's Philox4_32_10) and stores its
output.  Usage: python tests/golden/gen_philox_curand.py [out.json]"""
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main():
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "philox_curand.json"
    with tempfile.TemporaryDirectory() as td:
        exe = Path(td) / "gen"
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-o", str(exe),
                        str(HERE / "philox_curand.cu")], check=True)
        res = subprocess.run([str(exe)], check=True, capture_output=True, text=True)
    out.write_text(res.stdout)
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
