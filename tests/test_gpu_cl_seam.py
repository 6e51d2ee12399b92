"""The reference's own generation pipeline driving this engine through its GPU plug-in seam:
the reference sources built with -DUSE_OPENCL (src/generate.c:303-548; src/cl_generate.c
left out) and linked to libcablegen_b200_cl.so, whose cl_* functions (include/cablegen_cl.h,
inc/cl_generate.h:16-63) run the moves and spawns on the GPU while the reference merges the
sorted results on the CPU.  The layer files must hash to the reference CPU build's, and the
run must not fall back to the CPU path."""
import os
import subprocess
import sys

import pytest

from helpers import GOLDEN, ROOT, digests

sys.path.insert(0, GOLDEN)
from make_golden import prepare, sha  # noqa: E402

pytestmark = pytest.mark.gpu

CLI_CL = os.path.join(ROOT, "oracle", "_ref", "cli_cl")
FALLBACK = ("falling back", "failed; running CPU", "OpenCL move failed", "OpenCL spawn failed")


@pytest.mark.parametrize("name,end", [("plain_2x4_nearwall", None), ("ll_pruned", 120)])
def test_reference_pipeline_on_cuda_seam(tmp_path, name, end):
    if not os.path.exists(CLI_CL):
        pytest.skip("cli_cl is built only where the reference sources exist (make -C oracle ref_cl)")
    wl, form, conf, bdir, tdir = prepare(name, end, str(tmp_path), 4)
    with open(conf) as f:
        text = f.read().replace("use_gpu = false", "use_gpu = true")
    with open(conf, "w") as f:
        f.write(text)
    r = subprocess.run([CLI_CL, f"-C={conf}", "generate"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=900, env=dict(os.environ, XDG_CONFIG_HOME=str(tmp_path)))
    log = r.stdout + r.stderr
    assert r.returncode == 0, log[-3000:]
    assert not any(w in log for w in FALLBACK), [l for l in log.splitlines() if any(w in l for w in FALLBACK)][:5]
    want = digests(name)["layers"]
    last = form.end_gen
    for s in range(form.start, last + 1, 2):
        assert sha(os.path.join(bdir, f"{s}.boards")) == want[str(s)]["boards_sha256"], s
