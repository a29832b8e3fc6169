"""Command lines of the reference package (``nlo-bk``, ``nlo-dis``) on the device path.

Run them as ``python -m nlo_bk_optimized_b200.cli.nlobk`` and
``python -m nlo_bk_optimized_b200.cli.nlodis``.
"""
