"""Command-line text exports of a flat CSR, in place of the reference's
converters (tools/bin2ligra.cpp, bin2ligraweight.cpp, bin2totem.cpp,
bin2totemweight.cpp), which take the file prefix as their only argument:

    python -m scaph_b200.export bin2ligra <prefix>        # -> <prefix>.ligra
    python -m scaph_b200.export bin2ligraweight <prefix>  # -> <prefix>.ligra.weight
    python -m scaph_b200.export bin2totem <prefix>        # -> <prefix>.totem
    python -m scaph_b200.export bin2totemweight <prefix>  # -> <prefix>weight.totem
"""
from __future__ import annotations

import sys

import scaph_b200 as S

TOOLS = {"bin2ligra": S.EXPORT_LIGRA, "bin2ligraweight": S.EXPORT_LIGRA_WEIGHT,
         "bin2totem": S.EXPORT_TOTEM, "bin2totemweight": S.EXPORT_TOTEM_WEIGHT}


def main(argv: list[str]) -> int:
    if len(argv) != 2 or argv[0] not in TOOLS:
        print(__doc__.strip(), file=sys.stderr)
        return 2
    print(S.csr_export(argv[1], TOOLS[argv[0]]))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
