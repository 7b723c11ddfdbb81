"""The phase probe's host side on the CPU.  The probe build of the library
adds clock64() marks into 32 counters per CTA (slot 31 counts the ticks);
the driver's tables name the slots the kernels mark.  Checked here: the
tables stay inside the counters and clear of the tick count, the two groups
of the ProcUpdLazy tick use disjoint slots, the ProcUpdMulti table names
slots 0-12 of its resident launch, and the driver refuses the default build,
which has no probe counters."""
import os
import subprocess
import sys

from gsbn_b200 import phase_probe

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SLOTS, TICKS = 32, 31


def test_tables_inside_the_counters():
    for table in (phase_probe.PHASES_A, phase_probe.PHASES_B, phase_probe.PHASES_MULTI):
        assert all(0 <= k < SLOTS and k != TICKS for k in table)
        assert len(set(table.values())) == len(table)


def test_lazy_groups_use_disjoint_slots():
    assert not set(phase_probe.PHASES_A) & set(phase_probe.PHASES_B)


def test_multi_table_names_the_resident_slots():
    assert sorted(phase_probe.PHASES_MULTI) == list(range(13))


def test_refuses_the_default_build():
    env = dict(os.environ)
    env.pop("GSBN_B200_LIB", None)
    r = subprocess.run([sys.executable, "-m", "gsbn_b200.phase_probe"], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode != 0
    assert "phase-probe build" in r.stderr
