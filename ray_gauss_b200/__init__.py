"""B200-native (sm_100a) engine for RayGauss's differentiable volumetric Gaussian ray caster.

The torch-level drop-in is :mod:`ray_gauss_b200.optix_raycasting.render_optix`
(``RenderOptixFunction``, ``RenderOptixSettings``); :mod:`ray_gauss_b200.batched` renders many
views per launch; :mod:`ray_gauss_b200.engine` wraps the C ABI declared in
``include/raygauss_b200.h``.  Around the renderer: :mod:`ray_gauss_b200.graph` (the step as one
CUDA graph), :mod:`ray_gauss_b200.train_tail` (fused Adam / statistics / clamps, the ``get_data``
activations, schedules and optimizer-state surgery), :mod:`ray_gauss_b200.densify`,
:mod:`ray_gauss_b200.io` (PLY and checkpoints), :mod:`ray_gauss_b200.filter3d`,
:mod:`ray_gauss_b200.knn` and :mod:`ray_gauss_b200.losses`.
"""
__version__ = "0.1.0"
