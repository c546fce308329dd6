"""bench.py's host-side legs on small cases, on the CPU: the CPU baseline's state (the whole beach, the
ridge's slab sample split as the device splits) and the reference arm's JSON line."""
import argparse
import contextlib
import io
import json

import numpy as np

import bench
from pysurf_b200 import cases


def test_the_cpu_state_of_the_beach_is_the_whole_case():
    case = cases.solitaryBeach(8)
    state, fluid, what = bench.cpuState(case, False)
    assert fluid == case.fluidCount and len(state['positions']) == case.state.nParticles
    assert 'whole case' in what


def test_the_ridge_sample_is_a_split_slab_of_whole_columns():
    case = cases.ridgeWave3D(6)
    state, fluid, what = bench.cpuState(case, True)
    x = state['positions']
    assert fluid == int(state['isFluid'].sum()) > 0
    assert np.abs(x[:, 1] - 0.5 * case.info['tank'][1]).max() < 0.125 + case.spacing
    # the split's daughters are there, with an eighth of the mass and half the length
    assert (state['lengths'] < case.smoothingLength).any()
    assert state['masses'].sum() > 0 and np.isfinite(state['neighbours'])
    assert 'crest zone split' in what


def test_the_reference_arm_prints_its_line():
    args = argparse.Namespace(gpus=1, steps=2, warmup=1, impl='reference', case='beach', ppd=8, no_refine=False,
                              options='')
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.referenceArm(args)
    line = json.loads(out.getvalue().strip().splitlines()[-1])
    assert line['impl'] == 'reference' and line['value'] > 0 and line['unit'] == 'particle-updates/s'
    assert line['cpu_baseline']['kind'] == 'port' and line['e2e']['h2d_bytes_per_step'] == 0
