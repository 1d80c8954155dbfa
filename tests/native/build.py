"""Builds tests/native/libplan_emulator.so (test-only host emulator of the
engine's fusion plans) from the planner sources in snuqs_b200/csrc."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(os.path.dirname(HERE)), "snuqs_b200", "csrc")
OUT = os.path.join(HERE, "libplan_emulator.so")
SRCS = [os.path.join(HERE, "plan_emulator.cc"), os.path.join(CSRC, "gates.cc"),
        os.path.join(CSRC, "planner.cc"), os.path.join(CSRC, "adjoint_plan.cc")]


def build() -> str:
    deps = SRCS + [os.path.join(CSRC, f) for f in ("host_ops.h", "sq_plan.h", "adjoint_plan.h")]
    if not os.path.exists(OUT) or any(os.path.getmtime(s) > os.path.getmtime(OUT) for s in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC,
                        "-include", "algorithm", *SRCS, "-o", OUT], check=True)
    return OUT


if __name__ == "__main__":
    print(build())
