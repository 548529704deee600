"""B200-native direct-SCF J/K engine with the call interface of ByteQC's
``cuobc`` get_jk path."""
__version__ = '0.1.0'
