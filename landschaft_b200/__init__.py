"""landschaft_b200: landschaft's Omniscape moving-window circuit connectivity on one B200.

``omniscape`` is the drop-in for ``landschaft.omniscape`` (same arguments and
outputs); the windows are solved by hand-written sm_100a CUDA behind the C ABI
of ``include/lsb_omniscape.h``.
"""

from .omni import (  # noqa: F401
    Dataset,
    make_params,
    omniscape,
    omniscape_correction,
    read_reclass_table,
    reclassify,
    run_device,
    source_from_resistance,
)

from .autograd import grad_device, omniscape_current  # noqa: F401,E402
from .tune import autotune, clear_tuning, load_tuning, save_tuning, tuning_table  # noqa: F401,E402
from .raster import AdvancedResult, advanced, advanced_batch  # noqa: F401,E402
from .ini import omniscape_ini, parse_ini, read_ascii_grid, write_ascii_grid  # noqa: F401,E402

__version__ = "0.1.0"
