"""Import alias so code written against the reference (``from cusoap import
SOAP``) runs on the B200 implementation unchanged."""
from cusoap_b200 import SOAP

__all__ = ["SOAP"]
__version__ = "0.1.0"
