"""Real FFT objects (the ``janus.fft`` package of the reference).

Planner flags are accepted with FFTW's public values for interface parity
(janus/fft/__init__.py:64-72, janus/fft/serial/_serial_fft.pyx:10-18).  The
radix schedule of each axis is fixed by its length; the planning rigour
instead selects how a Green operator built on the transform
(``janus_b200.green``, ``transform=``) schedules its column passes on first
use: FFTW_ESTIMATE the built-in rule; FFTW_MEASURE (the default) and
FFTW_WISDOM_ONLY the autotuner's cached schedule for the grid when there is
one ("wisdom"), else the rule; FFTW_PATIENT and FFTW_EXHAUSTIVE run the
autotuner (timed candidates) and cache its choice.
"""
from .serial import (FFTW_CONSERVE_MEMORY, FFTW_DESTROY_INPUT, FFTW_ESTIMATE,
                     FFTW_EXHAUSTIVE, FFTW_MEASURE, FFTW_PATIENT,
                     FFTW_PRESERVE_INPUT, FFTW_UNALIGNED, FFTW_WISDOM_ONLY)

__all__ = ["FFTW_ESTIMATE", "FFTW_MEASURE", "FFTW_PATIENT", "FFTW_EXHAUSTIVE",
           "FFTW_WISDOM_ONLY", "FFTW_DESTROY_INPUT", "FFTW_PRESERVE_INPUT",
           "FFTW_UNALIGNED", "FFTW_CONSERVE_MEMORY"]
