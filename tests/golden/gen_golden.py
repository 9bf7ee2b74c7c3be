#!/usr/bin/env python
"""Generate the golden fixtures from the reference library itself.

Run in a container that has the reference sources, with FAF_REFERENCE_SRC
pointing at them:

    FAF_REFERENCE_SRC=<reference source tree> python tests/golden/gen_golden.py

It builds the reference (oracle/Makefile `ref` target) if needed, runs every
case of cases.py through the reference's public API (oracle/ref_driver.c ->
faf_execute / chirp_compile), and writes
  golden.npz      reference outputs (float32) for the seeded inputs
  policy.json     faf_is_size_supported / faf_get_recommended_size / create
                  error messages of the reference
  abi.json        field offsets, struct sizes and enum values compiled from
                  the reference's include/fastandfourier.h
The GPU host has no reference sources; the tests read only these files.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases  # noqa: E402
from oracle import refimpl  # noqa: E402

REF_INCLUDE = os.path.join(refimpl.REFERENCE_SRC, "include")

ABI_PROGRAM = r"""
#include <stdio.h>
#include <stddef.h>
#include "fastandfourier.h"
#define OFF(T, f) printf("\"%s.%s\": %zu,\n", #T, #f, offsetof(T, f))
int main(void) {
  printf("{\n");
  OFF(faf_config, n); OFF(faf_config, precision); OFF(faf_config, layout);
  OFF(faf_config, norm); OFF(faf_config, dir); OFF(faf_config, backend);
  OFF(faf_config, flags); OFF(faf_config, family); OFF(faf_config, levels);
  OFF(faf_config, conv); OFF(faf_config, dwt_backend); OFF(faf_config, dct_type);
  OFF(faf_config, hop_length); OFF(faf_config, win_length);
  OFF(faf_buffer, re); OFF(faf_buffer, im); OFF(faf_buffer, n); OFF(faf_buffer, layout);
  OFF(faf_transform, n); OFF(faf_transform, n_inst); OFF(faf_transform, code);
  OFF(faf_transform, twiddles); OFF(faf_transform, twiddle_sizes);
  OFF(faf_transform, precision); OFF(faf_transform, type); OFF(faf_transform, flags);
  OFF(faf_transform, jit_cache); OFF(faf_transform, hop_length);
  OFF(faf_transform, win_length); OFF(faf_transform, levels); OFF(faf_transform, family);
  OFF(faf_transform, cfg); OFF(faf_transform, scratch); OFF(faf_transform, scratch_size);
  OFF(faf_transform, execute_func); OFF(faf_transform, inner); OFF(faf_transform, inner_inv);
  OFF(faf_transform, user_aux); OFF(faf_transform, user_aux_im);
  OFF(faf_transform, user_aux_n); OFF(faf_transform, custom_h); OFF(faf_transform, custom_g);
  OFF(faf_transform, custom_ht); OFF(faf_transform, custom_gt);
  OFF(faf_transform, custom_len_hg); OFF(faf_transform, custom_len_syn);
  printf("\"sizeof.faf_config\": %zu,\n", sizeof(faf_config));
  printf("\"sizeof.faf_buffer\": %zu,\n", sizeof(faf_buffer));
  printf("\"sizeof.faf_inst\": %zu,\n", sizeof(faf_inst));
  printf("\"enum.FAF_TRANSFORM_PIPELINE\": %d,\n", (int)FAF_TRANSFORM_PIPELINE);
  printf("\"enum.FAF_TRANSFORM_STFT\": %d,\n", (int)FAF_TRANSFORM_STFT);
  printf("\"enum.FAF_LAYOUT_INTERLEAVED\": %d,\n", (int)FAF_LAYOUT_INTERLEAVED);
  printf("\"enum.FAF_NORM_FORWARD\": %d,\n", (int)FAF_NORM_FORWARD);
  printf("\"enum.FAF_BACKEND_JIT\": %d,\n", (int)FAF_BACKEND_JIT);
  printf("\"enum.FAF_CALL_BUILTIN\": %d,\n", (int)FAF_CALL_BUILTIN);
  printf("\"enum.FAF_FLAG_BLUESTEIN\": %u,\n", (unsigned)FAF_FLAG_BLUESTEIN);
  printf("\"enum.FAF_FLAG_MEASURE\": %u\n", (unsigned)FAF_FLAG_MEASURE);
  printf("}\n");
  return 0;
}
"""


def abi_offsets(include_dir):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "abi.c")
        exe = os.path.join(d, "abi")
        with open(src, "w") as f:
            f.write(ABI_PROGRAM)
        subprocess.run(["gcc", "-std=c11", "-I", include_dir, src, "-o", exe], check=True)
        return json.loads(subprocess.run([exe], capture_output=True, text=True, check=True).stdout)


def main():
    if not refimpl.sources_present():
        sys.exit("gen_golden: set FAF_REFERENCE_SRC to the reference's source tree")
    if not refimpl.available():
        refimpl.build()
    out = {}
    for n in cases.C2C_SIZES + cases.RADER:
        re, im = cases.c2c_input(n)
        for inv in (0, 1):
            yr, yi = refimpl.c2c(re, im, inverse=inv)
            out[f"c2c_{n}_{inv}"] = np.stack([yr, yi])
    for n in cases.BLUESTEIN:
        re, im = cases.c2c_input(n)
        for inv in (0, 1):
            yr, yi = refimpl.c2c(re, im, inverse=inv, flags=cases.FLAG_BLUESTEIN)
            out[f"blue_{n}_{inv}"] = np.stack([yr, yi])
    for n in cases.BIG_C2C:
        re, im = cases.c2c_input(n, batch=1)
        yr, yi = refimpl.c2c(re, im)
        out[f"c2c_{n}_0"] = np.stack([yr, yi])
    for n in cases.REAL_SIZES:
        x = cases.real_input(n)
        Xr, Xi = refimpl.r2c(x)
        out[f"r2c_{n}"] = np.stack([Xr, Xi])
        out[f"c2r_{n}"] = refimpl.c2r(Xr, Xi, n)
    for key, src, ops, n in cases.PIPELINES:
        x = cases.notch_signal(n=n) if key == "pipe_notch4096" else cases.real_input(n, seed=7)
        if ops == "mask":
            m = cases.notch_mask(n)
            out[key] = refimpl.pipeline(src, x, m, np.zeros_like(m))
        else:
            out[key] = refimpl.pipeline(src, x)
    n, win, hop, L = cases.STFT
    xs = cases.real_input(L, batch=2, seed=4)
    Xr, Xi = refimpl.stft(xs, n, win, hop)
    out["stft"] = np.stack([Xr, Xi])
    for n in cases.CWT:
        psi, _ = refimpl.cwt_bank(n)
        out[f"cwt_psi_{n}"] = psi
        out[f"cwt_{n}"] = refimpl.cwt(cases.real_input(n, batch=1, seed=9))
        # the inverses of those coefficients, and the L1 inverse's constants
        out[f"icwt_dual_{n}"] = refimpl.icwt(out[f"cwt_{n}"], 0)
        out[f"icwt_l1_{n}"] = refimpl.icwt(out[f"cwt_{n}"], 1)
        out[f"cwt_consts_{n}"] = np.array(refimpl.cwt_consts(n), np.float64)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)

    policy = {"supported": {}, "recommended": {}, "create": []}
    for t in (0, 2):
        policy["supported"][str(t)] = [int(refimpl.is_size_supported(t, n)) for n in cases.POLICY_N]
        policy["recommended"][str(t)] = [refimpl.recommended_size(t, n) for n in cases.POLICY_N]
    for t, n, fl in cases.CREATE_PROBES:
        ok, msg = refimpl.try_create(t, n, fl)
        policy["create"].append({"type": t, "n": n, "flags": fl, "ok": ok, "error": msg})
    policy["n"] = cases.POLICY_N
    with open(os.path.join(HERE, "policy.json"), "w") as f:
        json.dump(policy, f, indent=1)
    with open(os.path.join(HERE, "abi.json"), "w") as f:
        json.dump(abi_offsets(REF_INCLUDE), f, indent=1, sort_keys=True)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
