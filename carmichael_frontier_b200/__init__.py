"""B200-native exchange meet-in-the-middle residue join (k=64 Carmichael search).

Public surface:
  solve(M, Q, B0, r, B)        -> SolveResult with certified Carmichael hits
  solve_many([(M, Q, B0, r, B), ...]) -> one SolveResult each, solves overlapped with host work
  Solver                       -> reusable device state for repeated solves
  mitm_gpu2                    -> drop-in for the reference's gpu/mitm_gpu2.py
  workloads                    -> seeded instances with the benchmark shapes
"""
from .solve import Hit, Instance, SolveResult, Solver, Tuning, solve, solve_many  # noqa: F401

__all__ = ["solve", "solve_many", "Solver", "SolveResult", "Hit", "Instance", "Tuning"]
