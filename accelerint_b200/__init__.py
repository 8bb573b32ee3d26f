"""accelerint_b200: batched stiff-ODE integration on one B200 behind accelerInt's C interface."""
