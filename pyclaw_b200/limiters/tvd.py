"""Limiter codes understood by the wave limiter (src/pyclaw/limiters/tvd.py:74-77;
philim.f90:19-32 adds Beam-Warming as 5)."""
minmod = 1
superbee = 2
vanleer = 3
MC = 4
beam_warming = 5
