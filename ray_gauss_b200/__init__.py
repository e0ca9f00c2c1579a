"""B200-native (sm_100a) engine for RayGauss's differentiable volumetric Gaussian ray caster.

The torch-level drop-in is :mod:`ray_gauss_b200.optix_raycasting.render_optix`
(``RenderOptixFunction``, ``RenderOptixSettings``); :mod:`ray_gauss_b200.batched` renders many
views per launch; :mod:`ray_gauss_b200.engine` wraps the C ABI declared in
``include/raygauss_b200.h``.
"""
__version__ = "0.1.0"
