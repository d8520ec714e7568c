"""Random seeds for runs (api/seed_generator.hpp: a std::random_device source;
the default seed is std::mt19937's, 5489)."""

import secrets


class SeedGenerator:
    def get(self):
        return secrets.randbits(32)

    @staticmethod
    def default_seed():
        return 5489
