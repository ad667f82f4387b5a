"""CPU timing harness for the reference's NTF iteration (test / baseline
infrastructure only; used by bench.py's cpu_baseline and --impl reference legs).

What is timed is the reference's OWN code: the AUNTF subclass for the
algorithm (ntf/auntf.hpp with ntf/ntf{mu,hals,anlsbpp}.hpp, the dimension
tree of dimtree/ddt.hpp) compiled unmodified into oracle/_ref/libref_planc.so,
driven as a library user drives it (dim_tree(true) before reset(initial
factors), compute_error(true), computeNTF() one outer iteration per step).
The tensor is a planc::Tensor of the reference holding the synthetic CP
workload, made on the host by the oracle's generator (the same function of
factors, noise level and seed as the GPU library's generator). BLAS threads
come from OPENBLAS_NUM_THREADS, OpenMP threads from OMP_NUM_THREADS; the
dimension tree runs the 16 threads its constructor fixes (ddt.hpp:53).

When the reference build is absent, the oracle's restatement of the same loop
(ntf_oracle.cpp) is timed instead ("port").
"""
import time

import numpy as np

from . import RefNTF, RefTensor, ntf_run, ref_available, synth_cp


def make_tensor(dims, A, sigma, seed, round_f32=True):
    """The synthetic workload as a reference planc::Tensor (Tensor(dims,
    data) over a host buffer that is released afterwards)."""
    X = synth_cp(dims, A, sigma, seed, clip=True, round_f32=round_f32)
    t = RefTensor(X)
    del X
    return t


def time_reference(tensor, F0, algo, warmup, steps, compute_error=True):
    """Times `steps` outer iterations of the reference's AUNTF after `warmup`
    untimed ones. Returns (seconds of each step, last relative error)."""
    s = RefNTF(tensor, F0, algo, dimtree=True, compute_error=compute_error)
    try:
        for _ in range(warmup):
            s.run(1)
        times, err = [], None
        for _ in range(steps):
            t0 = time.perf_counter()
            err = s.run(1)
            times.append(time.perf_counter() - t0)
    finally:
        s.close()
    return times, err


def time_port(dims, A, sigma, seed, F0, algo, warmup, steps, compute_error=True):
    """The oracle's restatement of the loop, for trees without the reference
    build. Returns (seconds per step, repeated per step; last error)."""
    X = synth_cp(dims, A, sigma, seed, clip=True, round_f32=True)
    if warmup:
        ntf_run(X, F0, algo, warmup, dimtree=True, compute_error=compute_error)
    t0 = time.perf_counter()
    _, _, errs = ntf_run(X, F0, algo, steps, dimtree=True, compute_error=compute_error)
    dt = (time.perf_counter() - t0) / max(steps, 1)
    return [dt] * steps, float(errs[-1]) if compute_error else None


def run(dims, A, sigma, seed, F0, algo, warmup, steps, compute_error=True):
    """Times the reference (or the port) on the full workload. Returns a dict:
    kind, seconds per step, last error, set-up seconds."""
    t0 = time.perf_counter()
    if ref_available():
        t = make_tensor(dims, A, sigma, seed)
        setup = time.perf_counter() - t0
        try:
            times, err = time_reference(t, F0, algo, warmup, steps, compute_error)
        finally:
            t.close()
        kind = "reference"
    else:
        times, err = time_port(dims, A, sigma, seed, F0, algo, warmup, steps, compute_error)
        setup = 0.0
        kind = "port"
    return {"kind": kind, "step_s": times, "error": err, "setup_s": setup}
