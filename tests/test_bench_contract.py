"""bench.py's CPU reference arm stays CPU-only: it must not import the
package or load the GPU library (its timing would then not be the
reference's alone), and it reports the same `config` as the GPU arm."""

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_loads_no_gpu_library():
    code = (
        "import sys; sys.path.insert(0, %r); import bench; bench._ref_setup(); "
        "assert not [m for m in sys.modules if m.startswith('spyker_b200')], 'package imported'; "
        "maps = open('/proc/self/maps').read(); assert 'libspyker_b200' not in maps, 'GPU library loaded'; "
        "assert bench.headline_config(4096, 1) == bench.headline_config(4096, 1); print('ok')" % ROOT
    )
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr[-2000:]
