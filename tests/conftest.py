import json
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, 'tests', 'golden')
for p in (os.path.join(REPO, 'srdatalog-python_b200'), os.path.join(REPO, 'oracle'), GOLDEN, REPO):
  if p not in sys.path:
    sys.path.insert(0, p)


def pytest_configure(config):
  config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (runs on the B200 box)')


def load_plan(name: str) -> dict:
  with open(os.path.join(GOLDEN, 'plans', f'{name}.json')) as f:
    return json.load(f)


@pytest.fixture(scope='session')
def plans():
  return {n: load_plan(n) for n in ('tc', 'sg', 'triangle', 'tc_left', 'tc_lsm')}


@pytest.fixture(scope='session')
def expected():
  with open(os.path.join(GOLDEN, 'expected.json')) as f:
    return json.load(f)
