"""Persistence of autotuner choices: a JSON file mapping a key (GPU name, mesh or
batch shape, what was tuned) to the schedule the library's autotuner picked
(igab_autotune / igab_batch_autotune), so a later run applies it without
re-timing."""
import json
import os


def gpu_name(device=0):
    import torch
    return torch.cuda.get_device_name(device)


def mesh_key(device, nelem, phys, what):
    return "%s|mesh|%s|%dx%dx%d|%d" % (gpu_name(device), phys, nelem[0], nelem[1], nelem[2], what)


def batch_key(device, sizes, what):
    n = len(sizes)
    tot = sum(a * b * c for a, b, c in sizes)
    h = 0
    for a, b, c in sizes:
        h = (h * 1000003 + a * 961 + b * 31 + c) % (1 << 61)
    return "%s|batch|%d|%d|%x|%d" % (gpu_name(device), n, tot, h, what)


def load(path):
    if not path or not os.path.exists(path):
        return {}
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store(path, key, value):
    if not path:
        return
    data = load(path)
    data[key] = value
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
