"""Seeded synthetic tensors used by the parity tests (small enough for the
CPU oracle to finish in seconds)."""
import functools

import splatt_synth as S


@functools.lru_cache(maxsize=None)
def small3():
    return S.uniform_tensor([60, 45, 30], 6000, seed=11)


@functools.lru_cache(maxsize=None)
def med3():
    return S.uniform_tensor([400, 300, 200], 60000, seed=12)


@functools.lru_cache(maxsize=None)
def small4():
    return S.uniform_tensor([20, 15, 12, 9], 5000, seed=13)


@functools.lru_cache(maxsize=None)
def small5():
    return S.uniform_tensor([9, 8, 7, 6, 5], 4000, seed=14)


@functools.lru_cache(maxsize=None)
def zipf3():
    return S.zipf_tensor([3000, 2000, 800], 40000, 1.2, seed=15)


@functools.lru_cache(maxsize=None)
def zipf4():
    return S.zipf_tensor([5000, 2000, 500, 100], 60000, 1.2, seed=16)


ALL = dict(small3=small3, med3=med3, small4=small4, small5=small5, zipf3=zipf3, zipf4=zipf4)
