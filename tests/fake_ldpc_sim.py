#!/usr/bin/env python3
"""Test double: the real ``ldpc_sim`` command line (ldpcb200.sim.main) with a deterministic stub in
place of the GPU engine, so the reference's run_simulation.py can drive it on a machine without a
GPU.  Frame i is in error when i % 997 == 0 (with 7 bit errors); every frame takes 5 iterations."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "tt-ldpc-qb2-sim_b200"))

from ldpcb200 import sim  # noqa: E402


class StubEngine:
    calls = []

    def __init__(self, mat, punctured, device):
        self.mat = mat

    def describe(self):
        return "stub engine"

    def run(self, o, mu, sigma, l_max, first, n):
        fe = len(range((first + 996) // 997 * 997, first + n, 997))
        StubEngine.calls.append((first, n))
        return sim.Batch(n, 7 * fe, fe, 5 * n, 0.0)

    def close(self):
        pass


if __name__ == "__main__":
    sys.exit(sim.main(engine_factory=StubEngine))
