"""B200-native engine for libgrpp's GRPP integral path (see include/libgrpp.h)."""
from .system import (CART_ORDER_DIRAC, CART_ORDER_TURBOMOLE, GRPP, Potential, Shell, System,
                     cartesian_list, ncart)

__all__ = ["CART_ORDER_DIRAC", "CART_ORDER_TURBOMOLE", "GRPP", "Potential", "Shell", "System",
           "cartesian_list", "ncart"]
