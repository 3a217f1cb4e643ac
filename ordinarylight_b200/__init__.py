"""B200-native wavefront path tracer for OrdinaryLight.

Public surface:

* :class:`CudaWavefrontRenderer` / :class:`CudaRendererConfig` — the
  ``renderers.cuda`` RendererImplementation (sm_100a kernels via the C ABI of
  ``libolcuda.so``, declared in ``include/olcuda.h``);
* :class:`Renderer` — the renderer-neutral facade (``renderer_preference="cuda"``);
* the scene model mirror (``Scene``, ``Material``, ``Texture``,
  ``Transform``, cameras, lights) for use without the reference package;
* ``CudaWavefrontRenderer.render_batch`` / ``submit`` / ``serve_step`` and
  :mod:`ordinarylight_b200.serving` — the batched and served forms of the
  same path; :mod:`ordinarylight_b200.autotune` and
  :mod:`ordinarylight_b200.distributed` around them.
"""

from .scene import (  # noqa: F401
    CAMERA_TYPES, LIGHT_TYPES, DirectionalLight, EnvironmentLight, Instance, Material, Mesh, MeshResource,
    OrthographicCamera, PanoramicCamera, PerspectiveCamera, PointLight, Scene, SpotLight, Texture, TextureTransform,
    Texture1D, Transform, Volume, VolumeMaterial,
)
from .renderer import Renderer, RenderJob, RenderStatistics, install_cuda_preference  # noqa: F401
from .renderers.cuda import CudaRendererConfig, CudaWavefrontRenderer  # noqa: F401

__version__ = "0.1.0"
