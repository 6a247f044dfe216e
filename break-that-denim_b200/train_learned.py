"""Trains the learned coarse correction's network on the GPU and writes its weights next to this file
(learned_coarse.f32, float32, the flat layout of btd.h's btd_set_learned).

The material is logged on the device by the plain solver itself (coarsest operators and residuals of
every V-cycle) over the configurations' scenes, whitened and solved exactly on the device, and the
network is trained there by the library's BF16 forward and backward kernels with Adam
(learned.train_network). Needs a CUDA device.

Usage: python break-that-denim_b200/train_learned.py [--steps 1500] [--seed 0] [--out PATH]
"""
import argparse
import importlib.util
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def package():
    if "btd_b200" in sys.modules:
        return sys.modules["btd_b200"]
    spec = importlib.util.spec_from_file_location("btd_b200", os.path.join(HERE, "__init__.py"), submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["btd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    btd = package()
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=btd.learned.DEFAULT_PATH)
    args = ap.parse_args()
    t = time.time()
    w, hist = btd.learned.train_network(steps=args.steps, seed=args.seed)
    print("loss every 100 steps:", " ".join(f"{float(hist[k:k + 100].mean()):.3f}" for k in range(0, len(hist), 100)),
          f"({time.time() - t:.1f} s)", flush=True)
    btd.learned.save(w, args.out)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
