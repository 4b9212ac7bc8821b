"""B200 (sm_100a) JPEG 2000 decode pipeline with ThousandthChicken's stage
surface: CoefficientCoder, Quantizer, DWT (DWTForward53/97, DWTReverse53/97),
Preprocessor and Decoder, over the C ABI of libtc_j2k.so."""
from ._lib import LibraryMissing, TCError  # noqa: F401

__all__ = ["LibraryMissing", "TCError"]
