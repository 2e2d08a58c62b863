"""Two-electron integral entry points (mirror of ``ccsd_gpu.cuda``)."""
