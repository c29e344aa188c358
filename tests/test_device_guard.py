"""Every context-taking C-ABI entry point runs on the context's GPU.

CUDA's current device belongs to the host thread, and a thread that never
picked one runs on device 0. The table scheduler and the proof server call the
library from worker threads, so each entry point that takes an sg_ctx makes
the context's device current first (sg::enter in csrc/common.cuh). Checked here
without a GPU: (1) the guard's logic, compiled with g++ against a fake CUDA
runtime whose current device is per-thread, entered from fresh threads; (2)
every exported function of the library that takes a context (or a FRI state
that holds one) calls the guard before its first CUDA call."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "lambda_vm_b200", "csrc")
CHOST = os.path.join(ROOT, "tests", "c_host")


def test_worker_threads_enter_the_contexts_device(tmp_path):
    exe = str(tmp_path / "device_guard")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I" + os.path.join(CHOST, "fake_cuda"),
                        "-I" + os.path.join(ROOT, "include"), os.path.join(CHOST, "device_guard.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr


def _functions(src):
    """(name, params, body) of every top-level sg_* function definition."""
    out = []
    for m in re.finditer(r'^(?:extern "C" )?(?:int|void|uint64_t|uint32_t) (sg_\w+)\(([^)]*)\)\s*\{', src, re.M):
        end = src.find("\n}", m.end())
        out.append((m.group(1), m.group(2), src[m.end():end]))
    return out


# Entry points that take a context but never touch the device.
NO_CUDA = {"sg_ctx_launches", "sg_ctx_budget", "sg_ctx_fail_alloc_after", "sg_ctx_dft_tiles", "sg_ctx_memory",
           "sg_ctx_pass_log", "sg_ctx_set_pass_model"}


def test_every_context_entry_point_enters_its_device():
    checked, missing = [], []
    for fn in sorted(os.listdir(CSRC)):
        if not fn.endswith(".cu"):
            continue
        for name, params, body in _functions(open(os.path.join(CSRC, fn)).read()):
            takes_ctx = re.search(r"\bsg_ctx\s*\*\s*c\b", params)
            if not takes_ctx or name in NO_CUDA:
                continue
            checked.append(name)
            guard = re.search(r"SG_ENTER\(|\benter\(ctx\)", body)
            first_cuda = re.search(r"\bcuda[A-Z]\w*\(|<<<|dev_alloc\(|\b(?:coset_lde|ntt_rows|leaves_row_major|"
                                   r"merkle_inner|pad_leaves|fri_fold_step|launch_\w+)\(", body)
            if not guard or (first_cuda and first_cuda.start() < guard.start()):
                missing.append(f"{fn}:{name}")
    assert len(checked) >= 30, checked
    assert not missing, f"entry points that do not make the context's device current first: {missing}"
    # the FRI state carries its context: its fold steps enter it too
    rounds = open(os.path.join(CSRC, "rounds.cu")).read()
    step = rounds[rounds.index("static int fri_fold_step"):]
    step = step[:step.index("\n}")]
    assert "SG_ENTER(ctx)" in step and step.index("SG_ENTER(ctx)") < step.index("dev_alloc(")
