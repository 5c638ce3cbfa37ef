"""epigpu_b200 -- the exhaustive pairwise epistasis scan of epiGPU on NVIDIA B200 (sm_100a).

Native parts (built in-tree by `python -m epigpu_b200.build`):
  libepigpu.so  CUDA kernels behind the C ABI of include/epigpu.h
  bin/epiGPU    the C host program with epiGPU's -A command line and results file
Python modules: capi (ctypes binding), synth (seeded synthetic inputs),
epigpu_file (.epigpu reader/writer), results (results-file reader).
"""
