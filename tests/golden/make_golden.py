"""Extract the published FP64 golden finals from the reference's Benchmark.md.

Writes tests/golden/benchmark_finals.json: for each selected run (host, N, backend, FP64,
1 rank) the step count from the "Detailed Timing Records" block and the t = 20 diagnostics
from the "Final Diagnostic Records" block, with the source line numbers.  The runs are the
reference's adaptive-CFL Taylor-Green benchmark (CFL 0.5, dt cap 0.5, t_end 20, output_dt 1).

Run in a container that has the reference checked out (it is not read at test time):
    python tests/golden/make_golden.py /path/to/reference/Benchmark.md
"""
import json
import os
import re
import sys

RUNS = [("bobby", 64, "AVA(CPU)+FFTW"), ("lucia", 128, "AVA(CUDA)+cuFFT"), ("lucia", 256, "AVA(CUDA)+cuFFT")]
HEADER = re.compile(r"^### (\S+) / (\d+)\^3 / (\S+) / p(\d+) / MPI (\d+) / GPU (\d+)\s*$")


def parse(path):
    lines = open(path).read().splitlines()
    section, cur, out = None, None, {}
    for no, line in enumerate(lines, start=1):
        if line.startswith("## "):
            section = line[3:].strip()
            cur = None
            continue
        m = HEADER.match(line)
        if m:
            host, n, backend, prec, ranks = m.group(1), int(m.group(2)), m.group(3), int(m.group(4)), int(m.group(5))
            cur = (host, n, backend) if prec == 64 and ranks == 1 else None
            continue
        if cur is None or cur not in RUNS:
            continue
        rec = out.setdefault(cur, {"host": cur[0], "n": cur[1], "backend": cur[2], "source": {}})
        if section == "Detailed Timing Records" and line.startswith("- calls:"):
            rec["steps"] = int(re.search(r"step=(\d+)", line).group(1))
            rec["source"]["steps"] = f"Benchmark.md:{no}"
        elif section == "Final Diagnostic Records":
            for key in ("kinetic_energy", "dissipation", "enstrophy", "max_spectral_divergence", "max_velocity"):
                mm = re.search(key + r"=([0-9.eE+-]+)", line)
                if mm and key not in rec:
                    rec[key] = float(mm.group(1))
                    rec["source"][key] = f"Benchmark.md:{no}"
    return [out[r] for r in RUNS]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference's Benchmark.md>")
    src = sys.argv[1]
    data = {"what": "FP64 t = 20 finals of the reference's adaptive-CFL Taylor-Green benchmark "
                    "(CFL 0.5, dt cap 0.5, t_end 20, output_dt 1)", "runs": parse(src)}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "benchmark_finals.json")
    with open(dst, "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
    print(f"wrote {dst}")


if __name__ == "__main__":
    main()
