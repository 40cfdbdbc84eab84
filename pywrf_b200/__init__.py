"""pywrf_b200: B200-native (sm_100a) ARW integration step with PyWRF's call surface."""
__version__ = "0.1.0"
