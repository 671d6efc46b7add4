"""Build libplapack_b200.so in place (nvcc, sm_100a) with the csrc/ Makefile."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"], check=True)
    return os.path.join(HERE, "libplapack_b200.so")


if __name__ == "__main__":
    print(build())
