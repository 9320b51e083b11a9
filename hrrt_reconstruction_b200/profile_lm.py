"""A compact listmode case for profiling the histogram kernels.

Generates `--events` synthetic l64 events on the device (the benchmark's
generator: config-1 phantom LORs, 10 % delayed, a time tag per 1000 events),
then histograms them `--reps` times through each device path (direct
16-bit atomics, 32-bit counters, partitioned) into span-3 prompt and delayed
sinograms and prints the device time per call.  It holds the word stream
(8 bytes per event) and the two 16-bit sinograms (1.9 GB), so 1e8 events fit
a profiler capture of single launches.

    python hrrt_reconstruction_b200/profile_lm.py --events 1e8 --reps 1
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

PATHS = (("direct", 16), ("wide", 64), ("partitioned", 32))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--events", type=float, default=1e8)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--paths", default="direct,wide,partitioned")
    args = ap.parse_args()

    import torch
    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import listmode_synth as LS
    with H.Context(H.hrrt_geometry(span=3)) as c3:
        E = LS.expected_prompts(c3, seed=0)
    words = LS.synth_words(int(args.events), E, seed=0)
    del E
    torch.cuda.synchronize()
    with H.Listmode(3) as lm:
        ds = torch.zeros(lm.sino_size, dtype=torch.int16, device="cuda")
        dd = torch.zeros(lm.sino_size, dtype=torch.int16, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        want = args.paths.split(",")
        for name, flag in PATHS:
            if name not in want:
                continue
            ms = []
            for r in range(args.reps + 1):
                lm.reset_clock()
                st = lm.histogram_device(words.data_ptr(), words.numel(), ds.data_ptr(), dd.data_ptr(), flags=flag,
                                         stream=stream)
                if r > 0:
                    ms.append(st["ms"])
            print(f"{name:12s} {int(args.events)} events  " + " ".join(f"{m:.2f}" for m in ms) + " ms", flush=True)


if __name__ == "__main__":
    main()
