"""gtls_b200: B200-native Transit Least Squares search behind ``gtls(t, y).power()``."""
from .main import gtls  # noqa: F401
from .results import gtlsResult  # noqa: F401
