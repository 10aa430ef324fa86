"""Element table stand-in (only what the reference's UPF reader looks up)."""
chemical_symbols = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
                    "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar"]
atomic_numbers = {symbol: number for number, symbol in enumerate(chemical_symbols)}
