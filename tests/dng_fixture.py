"""Synthetic DNG writer for the ingest tests (shared with the benchmark)."""
from cpipe_b200.dng_synth import *  # noqa: F401,F403
from cpipe_b200.dng_synth import ASCII, LONG, SHORT, build_dng  # noqa: F401
