"""Host helpers with the reference's names (beamax utils/)."""
from .coeff_index import batch_data, compute_coeff_shapes, find_level, find_tensor_and_multiindex  # noqa: F401
from .arrays import extract_centered_box, rel_l2  # noqa: F401
from .interp import GridInterpolant, make_c_function_from_grid  # noqa: F401
