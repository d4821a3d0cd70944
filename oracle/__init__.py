"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the filter + back-projection path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import this
package, as the checker of the CUDA path; the product never imports, links or runs it.

It restates minirecast (ZYHuang216/Tomography-local-demo, package `minirecast/`)
function by function - each function cites the reference file:line it follows:
  bp.py       ctypes front of bp_oracle.c (recon.py:156-219, Numba kernels in C)
  filter.py   recon.py:34-104 filter path, preprocess.py, flexray/hdf5 raw correction
  geometry.py geometry.py:60-72, recon.py:70-82 and 225-283 plane helpers, stream.py order
  phantom.py  phantom.py analytic ellipsoid projector (fixture generator)
  recon.py    SliceReconstructor pipeline (recon.py:289-519) at FP32-store / FP64
  ls.py       few-view least-squares slice refinement (no reference counterpart)
  model.py    otsu_threshold of the volume consumer (model.py:18-29)
Parity of this restatement is pinned against golden vectors produced by the reference
itself (tests/golden/make_golden.py, fixtures in tests/golden/*.npz).
"""
