"""B200-native aerial-image engine (Abbe and Hopkins/SOCS imaging)."""
from .params import (ImageData, Numerics, PolarizationParameters, Projection, Scatter, Source,  # noqa: F401
                     SourceData)
