"""new_fgssjoin_b200 -- B200-native Jaccard set-similarity self-join.

Python host side of ``libfgss.so`` (C ABI in ``include/fgss.h``).  It mirrors
the reference project's host interface for the join path
(RafaelQuirino/new_fgssjoin):

=====================================  =============================================
reference (file:line)                  here
=====================================  =============================================
``ppjoin_format(path, verbose)``       ``ppjoin_format(path)`` / ``Sets.from_bin``
(src/fgssjoin/data.cu:31-126)          records in MEMORY order (file order reversed)
preprocess selfjoin <file> <q>         ``Context.tokenize(text, q=...)`` on the GPU
(src/preprocess_cli.cpp:222-358)
``prepare_data`` + ``inverted_index``  ``Context.selfjoin(sets, threshold)``
+ ``process_blocks``                   returns the pairs block.cu:184-197 prints,
(src/fgssjoin_cli.cu:86-100)           sorted by (q, s), and the reference's counters
=====================================  =============================================

Errors raise :class:`FgssError` carrying the library status (the reference
prints and calls ``exit(1)``, src/util.cu:43-49).  There is no CPU fallback:
every compute call goes through the CUDA library and fails loudly when it is
missing or no B200 is present.
"""
from .binding import (FgssError, Context, Sets, Pairs, ppjoin_format, lib_path, load_library, bounds_table, overlap_table,  # noqa: F401
                      METHOD_PLAIN, METHOD_BATCHED, BOUNDS_REFERENCE, BOUNDS_EXACT, EXPORTED_SYMBOLS)

__all__ = ["FgssError", "Context", "Sets", "Pairs", "ppjoin_format", "lib_path", "load_library", "bounds_table", "overlap_table",
           "METHOD_PLAIN", "METHOD_BATCHED", "BOUNDS_REFERENCE", "BOUNDS_EXACT", "EXPORTED_SYMBOLS"]
