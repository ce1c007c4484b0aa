"""Oracle package: the CPU checker (cj_oracle.c), the build recipe for it and
for the reference's own execute(), and their ctypes bindings. Test
infrastructure only; the product never imports it."""
