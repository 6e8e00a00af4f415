"""mmnorm_b200 -- B200 (sm_100a) near-field SAR backprojection fused with the mmWave
surface-normal vote, behind the call signatures of mmNorm's imaging step.

Modules:
  ops           device-resident tensor API (backproject, surface_normals)
  py_image_gpu  drop-in ``image_cuda`` (src/data_processing/cuda/py_image_gpu.py)
  py_sn_est_gpu drop-in ``normal_estimates_cuda`` (src/data_processing/cuda/py_sn_est_gpu.py)
  pipeline      one-call image + unit normals (image_processor.py:383-396)
  scenes        seeded synthetic point-scatterer scenes
  build         nvcc recipe for the in-tree library
"""
__version__ = "0.1.0"
