"""Mirrors of the reference's engine_core Python API for the classic
build/lookup path (engine_core/BookBuilder.py, BookReader.py, Calculator.py),
running on libegtb_gpu."""
