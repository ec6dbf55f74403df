"""Legacy six-dimensional square game (src/pursuit_evasion/dp): grid,
solver on the GPU and the portable table reader."""
