"""bench.py's reference arm runs on the CPU and prints the one-line JSON contract (no GPU needed)."""
import json
import os
import subprocess
import sys

from conftest import REPO


def test_reference_arm_prints_the_contract_line():
    env = dict(os.environ, NUMBA_NUM_THREADS=str(min(4, os.cpu_count() or 1)))
    r = subprocess.run([sys.executable, os.path.join(REPO, 'bench.py'), '--impl', 'reference', '--steps', '2',
                        '--warmup', '1', '--ref-targets', '256'], capture_output=True, text=True, timeout=600,
                       env=env, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith('{')]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'scaling',
                'vs_baseline', 'dtype', 'data', 'config', 'impl', 'cpu_baseline', 'e2e'):
        assert key in d, key
    assert d['impl'] == 'reference' and d['steps'] == 2 and d['value'] > 0
    assert d['e2e']['h2d_bytes_per_step'] == 0 and d['e2e']['value'] == d['value']
    assert d['cpu_baseline']['kind'] == 'port'
