"""Real FFT objects (the ``janus.fft`` package of the reference).

Planner flags are accepted with FFTW's public values for interface parity
(janus/fft/__init__.py:64-72, janus/fft/serial/_serial_fft.pyx:10-18).  The
GPU transforms ignore the planning-rigor flags: the radix schedule of each
axis is fixed at creation.
"""
from .serial import (FFTW_CONSERVE_MEMORY, FFTW_DESTROY_INPUT, FFTW_ESTIMATE,
                     FFTW_EXHAUSTIVE, FFTW_MEASURE, FFTW_PATIENT,
                     FFTW_PRESERVE_INPUT, FFTW_UNALIGNED, FFTW_WISDOM_ONLY)

__all__ = ["FFTW_ESTIMATE", "FFTW_MEASURE", "FFTW_PATIENT", "FFTW_EXHAUSTIVE",
           "FFTW_WISDOM_ONLY", "FFTW_DESTROY_INPUT", "FFTW_PRESERVE_INPUT",
           "FFTW_UNALIGNED", "FFTW_CONSERVE_MEMORY"]
