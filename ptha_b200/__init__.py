"""B200 (sm_100a) implementation of the SWALS shallow-water time-step hot path.

The product is ``libswalsgpu.so`` (CUDA + C ABI, include/swals_gpu.h); this
package builds it and mirrors SWALS's ``domain_type`` API on top of it.
"""
from ._lib import SwalsError  # noqa: F401
from .domain import Domain, STG, UH, VH, ELV  # noqa: F401
from .multidomain import Multidomain, MultidomainGroup  # noqa: F401
from .nesting import NestDomain  # noqa: F401

__all__ = ["Domain", "Multidomain", "MultidomainGroup", "NestDomain", "SwalsError", "STG", "UH", "VH", "ELV"]
