"""Renderer implementations of ordinarylight_b200 (``renderers.cuda``)."""

from .base import RendererImplementation, RendererImplementationInfo, RendererProtocol  # noqa: F401
from .cuda import CudaRendererConfig, CudaWavefrontRenderer  # noqa: F401
