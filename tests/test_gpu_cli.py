"""The reference's own CLI (frontends/cli/main.c, parse.c), unmodified, linked against
libcablegen_b200.so: generate/solve files bit-exact, lookup/explore/read transcripts
identical to the reference CLI's, and the self-test passing."""
import os
import subprocess
import sys

import pytest

from helpers import GOLDEN, ROOT, digests

sys.path.insert(0, os.path.join(GOLDEN))
from make_golden import CLI_GAMES, CLI_WORKLOAD, cli_commands, cli_prepare, fixed_time_lib, run_game, sha  # noqa: E402

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "cablegen_b200", "_build", "cli_b200")


@pytest.fixture(scope="module")
def cli_dir(tmp_path_factory):
    if not os.path.exists(CLI):
        pytest.skip("cli_b200 is built only where the reference CLI sources exist")
    work = str(tmp_path_factory.mktemp("cli"))
    conf = cli_prepare(work)
    env = dict(os.environ, XDG_CONFIG_HOME=work)
    for c in ("generate", "solve"):
        r = subprocess.run([CLI, f"-C={conf}", c], cwd=work, env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
    return work, conf, env


def test_cli_files_match_reference(cli_dir):
    work, _, _ = cli_dir
    d = digests(CLI_WORKLOAD)["layers"]
    for s, rec in d.items():
        assert sha(os.path.join(work, "boards", f"{s}.boards")) == rec["boards_sha256"], s
        assert sha(os.path.join(work, "tables", f"{s}.tables")) == rec["tables_sha256"], s


@pytest.mark.parametrize("i", range(len(cli_commands())))
def test_cli_transcripts(cli_dir, i):
    work, conf, env = cli_dir
    cmd = cli_commands()[i]
    out = subprocess.run([CLI, f"-C={conf}"] + cmd, cwd=work, env=env, capture_output=True, text=True,
                         timeout=120).stdout
    with open(os.path.join(GOLDEN, "cli", f"{i:02d}_{cmd[0]}.txt")) as f:
        want = f.read()
    assert out == want


@pytest.mark.parametrize("game", CLI_GAMES, ids=[g[0] for g in CLI_GAMES])
def test_cli_play_and_train_transcripts(cli_dir, tmp_path, game):
    """play and train (frontends/cli/main.c:354-475) over this library's tables: with time()
    fixed (so srand seeds the same spawns) the transcript equals the reference CLI's."""
    work, conf, env = cli_dir
    cmd, board, stdin = game
    out = run_game(CLI, conf, work, env, cmd, board, stdin, fixed_time_lib(str(tmp_path)))
    with open(os.path.join(GOLDEN, "cli", f"game_{cmd}.txt")) as f:
        want = f.read()
    assert out == want


def test_cli_self_test(cli_dir):
    work, conf, env = cli_dir
    r = subprocess.run([CLI, f"-C={conf}", "test"], cwd=work, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "All tests passed!" in r.stdout


def test_cli_generate_resumes_from_checkpoint(tmp_path):
    """[Generate] checkpoint / resume (library extension): a generation stopped at tile sum 40
    and resumed up to 60 writes the same layer files as the reference."""
    if not os.path.exists(CLI):
        pytest.skip("cli_b200 is built only where the reference CLI sources exist")
    from make_golden import prepare
    work = str(tmp_path)
    wl, form, conf, bdir, tdir = prepare("ll_pruned", 40, work, 2)
    with open(conf) as f:
        text = f.read().replace("prune = true", "prune = true\ncheckpoint = true\nresume = true")
    env = dict(os.environ, XDG_CONFIG_HOME=work)

    def run(end):
        with open(conf, "w") as f:
            f.write(text.replace("end = 40", f"end = {end}", 1))
        r = subprocess.run([CLI, f"-C={conf}", "generate"], cwd=work, env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        return r.stdout + r.stderr

    first = run(40)
    assert "Resuming" not in first
    assert os.path.exists(os.path.join(bdir, "42.boards.resume"))
    for s in range(42, 61, 2):
        assert not os.path.exists(os.path.join(bdir, f"{s}.boards"))
    second = run(60)
    assert "Resuming at layer 42" in second
    assert os.path.exists(os.path.join(bdir, "62.boards.resume"))
    assert not os.path.exists(os.path.join(bdir, "42.boards.resume"))
    want = digests("ll_pruned")["layers"]
    for s in range(16, 61, 2):
        assert sha(os.path.join(bdir, f"{s}.boards")) == want[str(s)]["boards_sha256"], s
    assert "already generated" in run(60)
