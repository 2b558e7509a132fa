"""CPU checks of bench.py's reference arm, which times the oracle's float32 restatement of the reference
CPU path on the host cores: one JSON line with the contract's keys on rank 0, nothing (exit 0) on the
other ranks of a multi-rank launch."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_bench(*args, env=None):
    return subprocess.run([sys.executable, 'bench.py', *args], cwd=ROOT, capture_output=True, text=True,
                          timeout=900, env=env)


def test_reference_arm_prints_the_contract_line():
    out = run_bench('--impl', 'reference', '--steps', '1', '--warmup', '0')
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line['impl'] == 'reference'
    assert line['metric'].startswith('RTM shot-images/s') and line['unit'] == 'shot-images/s'
    assert line['value'] > 0 and line['higher_is_better'] is True and line['steps'] == 1
    assert line['cpu_baseline']['kind'] == 'port' and line['cpu_baseline']['cores'] >= 1
    assert line['cpu_baseline']['value'] == line['value']
    assert line['e2e'] == {'value': line['value'], 'unit': line['unit'], 'h2d_bytes_per_step': 0,
                           'd2h_bytes_per_step': 0}


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK='1', WORLD_SIZE='2')
    out = run_bench('--impl', 'reference', '--steps', '1', '--warmup', '0', env=env)
    assert out.returncode == 0 and out.stdout.strip() == ''
