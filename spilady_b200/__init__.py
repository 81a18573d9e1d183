"""B200-native spin-lattice dynamics step engine."""
