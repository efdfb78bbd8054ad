"""GeRaF RF operators on sm_100a: ``RFMatchedFilter`` and ``RFSignalTracer``."""
