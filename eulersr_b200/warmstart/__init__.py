"""Learned warm start: IDW interpolation of a coarse solution corrected by a
residual MLP, trained and run by the library's BF16 kernels."""
