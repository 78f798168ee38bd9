"""Package ``tcuscan``: re-exports ``tcuscan_ops`` exactly like the reference's
python/tcuscan/__init__.py:1-5 (import torch first, then the operators)."""
import torch  # noqa: F401

from tcuscan_ops import *  # noqa: F401,F403
